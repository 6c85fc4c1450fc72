"""One case split over two ranks whose right-hand sides run on the GPU.

Both ranks share the one GPU of the test machine and talk through gloo on
host memory: their kernels never wait on each other, only the host-side
collectives do.  ``src.domain.DomainSolver`` with ``EngineStepper``
(``mhd_rhs`` and the literal MHDStep stages through the C ABI) must give the
whole case's result: compared with the C oracle run in one process to FP64
rounding (each rank sums its neighbours in its own cell order).
"""

import datetime
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as tdist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from compare import assert_close, scales  # noqa: E402
from small_cases import blast_3d  # noqa: E402

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "u", "v", "w", "e", "h", "rho", "p", "cs", "Bx", "By", "Bz", "psi", "alpha1", "au",
          "av", "aw", "ae", "aBevolx", "aBevoly", "aBevolz", "apsi", "dt_adapt", "alphaloc", "divBsymm", "omega")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    ic, prm = blast_3d(n=20, seed=7)
    ic["u"] = ic["u"] + 2.0  # drift across the slab faces
    return ic, prm


def _worker(rank, world, port, steps, out_path):
    from src.domain import DomainSolver, EngineStepper
    from src.engine import params_from_dict

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        ic, prm = _case()
        arrays = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in ic.items()}
        share = slice(rank, None, world)  # an arbitrary first split; migration fixes it
        arrays = {k: v[share].contiguous() for k, v in arrays.items()}
        stepper = EngineStepper(params_from_dict(prm), capacity=len(ic["x"]))
        solver = DomainSolver(stepper, arrays, prm, axis=0)
        solver.warmup()
        dt = solver.initial_dt()
        for _ in range(steps):
            solver.step(dt)
            dt = solver.min_dt()
        out = solver.gather(FIELDS + ("gid",))
        ghosts = [None] * world
        tdist.all_gather_object(ghosts, sum(solver.ghost_counts))
        stepper.close()
        if rank == 0:
            np.savez(out_path, dt=dt, ghosts=np.array(ghosts), **out)
    finally:
        tdist.destroy_process_group()


def test_two_ranks_on_the_gpu_match_the_oracle(tmp_path):
    import oracle

    steps = 3
    ic, prm = _case()
    s = oracle.State(ic)
    o = oracle.Oracle(prm, exact_order=False)
    o.warmup(s)
    dt = o.initial_dt(s)
    for _ in range(steps):
        o.step(s, dt)
        dt = o.min_dt(s)
    ref = {k: s[k] for k in FIELDS}
    out = str(tmp_path / "r.npz")
    mp.spawn(_worker, args=(2, _free_port(), steps, out), nprocs=2, join=True)
    d = np.load(out)
    np.testing.assert_array_equal(d["gid"], np.arange(len(ic["x"]), dtype=np.float64))
    assert np.all(d["ghosts"] > 0)
    got = {k: d[k] for k in FIELDS}
    assert_close(got, ref, FIELDS, 1e-8, scales(ic, ref["cs"]), what="2 ranks vs oracle")
    assert abs(float(d["dt"]) - dt) <= 1e-9 * dt
