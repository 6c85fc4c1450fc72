"""The multi-rank path of the batched form, on CPU with the gloo backend.

Two ranks (processes) share out a batch of instances, each "advances" its
share with a CPU stand-in of the per-instance update (the GPU step itself is
covered by the single-GPU tests; nothing here needs a GPU), and the
collectives the benchmark uses -- barrier, max over ranks of the timed
region, gather of per-instance results -- must give what one process gives.
"""

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as tdist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _instance_result(k, size, steps):
    # deterministic stand-in for "advance instance k for `steps` steps"
    rng = np.random.default_rng(k)
    x = rng.random(size)
    for _ in range(steps):
        x = 0.5 * (x + np.roll(x, 1))
    return {"x": x}


def _worker(rank, world, port, sizes, steps, out_path):
    from src.parallel import checksum, gather_instances, max_over_ranks, shard_instances, sum_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        share = shard_instances(sizes, world)
        # every rank computed the same split
        seen = [None] * world
        tdist.all_gather_object(seen, share)
        assert all(s == share for s in seen)
        tdist.barrier()
        local = {k: checksum(_instance_result(k, sizes[k], steps)) for k in share[rank]}
        busy = float(sum(sizes[k] for k in share[rank]))
        longest = max_over_ranks(busy)
        total = sum_over_ranks(busy)
        merged = gather_instances(local, len(sizes))
        if rank == 0:
            np.savez(out_path, merged=np.array(merged), longest=longest, total=total,
                     loads=np.array([sum(sizes[k] for k in s) for s in share]))
    finally:
        tdist.destroy_process_group()


def test_shard_balances_and_covers_every_instance():
    from src.parallel import shard_instances

    rng = np.random.default_rng(0)
    sizes = (rng.integers(32, 257, 64) ** 2).tolist()
    for world in (1, 2, 3, 4, 8):
        share = shard_instances(sizes, world)
        assert sorted(k for s in share for k in s) == list(range(64))
        loads = [sum(sizes[k] for k in s) for s in share]
        # greedy largest-first: no rank exceeds the mean by more than the largest instance
        assert max(loads) - sum(loads) / world <= max(sizes)
        assert share == shard_instances(sizes, world)


def test_two_gloo_ranks_match_one_process(tmp_path):
    from src.parallel import checksum, gather_instances, shard_instances

    sizes = [500, 120, 333, 64, 900, 45, 210, 700, 81]
    steps = 5
    out = str(tmp_path / "r.npz")
    mp.spawn(_worker, args=(2, _free_port(), sizes, steps, out), nprocs=2, join=True)
    d = np.load(out)
    single = gather_instances({k: checksum(_instance_result(k, s, steps)) for k, s in enumerate(sizes)}, len(sizes))
    np.testing.assert_array_equal(d["merged"], np.array(single))
    loads = d["loads"]
    assert float(d["longest"]) == float(max(loads)) and float(d["total"]) == float(sum(sizes))
    assert list(loads) == [sum(sizes[k] for k in s) for s in shard_instances(sizes, 2)]


def test_gather_rejects_overlap_and_gaps():
    from src.parallel import gather_instances

    with pytest.raises(ValueError):
        gather_instances({0: 1.0}, 2)
