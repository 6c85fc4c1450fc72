"""Several GPUs, one process each: the batched form's instances shared out.

The per-instance update does not shard without a halo exchange per pair
pass, so one simulation stays on one GPU.  A batch of independent instances
does shard: every rank advances its own share of the instances with no
collective on the data path.  The collectives are the barrier around the
timed region, the max over ranks of its duration, and a gather of
per-instance results at the end.  They run on whatever process group is
initialised: NCCL on GPUs, gloo for the CPU tests.
"""

from __future__ import annotations

import numpy as np


def shard_instances(sizes, world: int):
    """Instance indices per rank, balancing particle counts: the largest
    instance first, each to the least loaded rank (ties to the lower rank).
    Deterministic, so every rank computes the same split; a rank's share is
    in ascending instance order."""
    sizes = [int(s) for s in sizes]
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    share = [[] for _ in range(world)]
    for k in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        r = min(range(world), key=lambda q: (load[q], q))
        share[r].append(k)
        load[r] += sizes[k]
    return [sorted(s) for s in share]


def _dist():
    import torch.distributed as tdist

    return tdist if tdist.is_available() and tdist.is_initialized() else None


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (the value itself without a group)."""
    tdist = _dist()
    if tdist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    tdist = _dist()
    if tdist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.SUM)
    return float(t.item())


def gather_instances(local: dict, n_inst: int):
    """Per-instance results {instance: value} of every rank merged into one
    list in instance order (on every rank).  Each instance must come from
    exactly one rank."""
    tdist = _dist()
    parts = [local]
    if tdist is not None:
        parts = [None] * tdist.get_world_size()
        tdist.all_gather_object(parts, local)
    out = [None] * n_inst
    for part in parts:
        for k, v in part.items():
            if out[k] is not None:
                raise ValueError(f"instance {k} came from two ranks")
            out[k] = v
    missing = [k for k, v in enumerate(out) if v is None]
    if missing:
        raise ValueError(f"instances {missing[:5]} came from no rank")
    return out


def checksum(arrays: dict) -> float:
    """An order-independent summary of an instance's final state (sum of
    squares over the given fields), for comparing sharded and single runs."""
    return float(sum(np.sum(np.asarray(v, dtype=np.float64) ** 2) for v in arrays.values()))
