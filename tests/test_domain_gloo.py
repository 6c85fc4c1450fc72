"""One case split over CPU ranks (gloo): slabs, migration and halos.

``src.domain.DomainSolver`` drives the warm-up, the initial step size and
PEC steps of one case whose particles are shared out over the ranks.  With
the C oracle as its stepper (``tests/domain_oracle.py``) the decomposed run
must equal a one-process oracle run bit for bit: every owned particle sees
exactly its whole-case neighbourhood, and every collective (min dt, max h,
migration, ghost exchange) gives what one process computes.  Particles are
given a drift along the split axis so that they cross slab faces during the
run, and rank 0 starts with every particle (the first migration shares them
out).
"""

import datetime
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as tdist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from small_cases import blast_3d, open_blob_2d, orszag_tang_2d  # noqa: E402

STATE = ("x", "y", "z", "u", "v", "w", "e", "h", "rho", "p", "cs", "Bx", "By", "Bz", "Bevolx", "Bevoly", "Bevolz",
         "psi", "alpha1", "alphaloc", "au", "av", "aw", "ae", "aBevolx", "aBevoly", "aBevolz", "apsi", "dt_adapt",
         "omega", "divBsymm")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(name):
    if name == "blast3d_x":
        ic, prm = blast_3d(n=16, seed=3)
        ic["u"] = ic["u"] + 2.0  # drift across the slab faces
        return ic, prm, 0
    if name == "orstang2d_y":
        ic, prm = orszag_tang_2d(n=36, seed=4)
        ic["v"] = ic["v"] + 1.5
        return ic, prm, 1
    ic, prm = open_blob_2d(n=40, seed=5)
    ic["u"] = ic["u"] + 0.5
    return ic, prm, 0


def _worker(rank, world, port, name, steps, out_path):
    from domain_oracle import OracleStepper, as_tensors
    from src.domain import DomainSolver

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        ic, prm, axis = _case(name)
        arrays = as_tensors(ic)
        if rank != 0:
            arrays = {k: v[:0] for k, v in arrays.items()}
        solver = DomainSolver(OracleStepper(prm, nthreads=1), arrays, prm, axis=axis)
        owned0 = int(solver.owned["x"].numel())
        solver.warmup()
        first = set(solver.owned["gid"].tolist())
        dt = solver.initial_dt()
        for _ in range(steps):
            solver.step(dt)
            dt = solver.min_dt()
        out = solver.gather(STATE + ("gid",))
        arrived = len(set(solver.owned["gid"].tolist()) - first)
        counts = [None] * world
        tdist.all_gather_object(counts, (owned0, int(solver.owned["x"].numel()), sum(solver.ghost_counts), arrived))
        if rank == 0:
            np.savez(out_path, dt=dt, counts=np.array(counts), redone=solver.redone, **out)
    finally:
        tdist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("blast3d_x", 2), ("orstang2d_y", 3), ("openblob2d_x", 2)])
def test_decomposed_run_equals_one_process(tmp_path, name, world):
    from domain_oracle import single_run

    steps = 4
    ic, prm, _ = _case(name)
    ref, dt_ref = single_run(ic, prm, steps)
    out = str(tmp_path / "r.npz")
    mp.spawn(_worker, args=(world, _free_port(), name, steps, out), nprocs=world, join=True)
    d = np.load(out)
    np.testing.assert_array_equal(d["gid"], ref["gid"])
    for k in STATE:
        np.testing.assert_array_equal(d[k], ref[k], err_msg=k)
    assert float(d["dt"]) == dt_ref
    counts = d["counts"]
    n = len(ic["x"])
    assert counts[:, 1].sum() == n
    # every rank owned a share and held ghosts; the shares are balanced
    assert counts[:, 1].min() > 0.5 * n / world and counts[:, 2].min() > 0
    # particles crossed slab faces during the steps and moved to their new owners
    assert counts[:, 3].sum() > 0
    # (in the open case the edge particles' h grows past the first halo, so a
    # step is redone with a wider one; the result is exact all the same)
    assert int(d["redone"]) <= 2


def test_slabs_owner_distance_and_balance():
    from src.domain import Comm, Slabs

    rng = np.random.default_rng(0)
    c = torch.from_numpy(rng.uniform(-0.5, 0.5, 10000) ** 3 * 4.0)
    s = Slabs.balanced(c, -0.5, 0.5, True, Comm(), bins=4096)
    assert s.world == 1 and s.cuts == [-0.5, 0.5]
    s = Slabs(-0.5, 0.5, True, [-0.5, -0.1, 0.2, 0.5])
    own = s.owner(torch.tensor([-0.5, -0.1000001, -0.1, 0.19, 0.2, 0.5], dtype=torch.float64))
    assert own.tolist() == [0, 0, 1, 1, 2, 2]
    # periodic distances through the wrap; zero inside
    d = s.distance(torch.tensor([0.45, -0.45, 0.0], dtype=torch.float64), 0)
    np.testing.assert_allclose(d.numpy(), [0.0 + 0.05, 0.0, 0.1], atol=1e-15)
    d2 = Slabs(-0.5, 0.5, False, [-0.5, -0.1, 0.2, 0.5]).distance(torch.tensor([0.45], dtype=torch.float64), 0)
    np.testing.assert_allclose(d2.numpy(), [0.55])
    with pytest.raises(ValueError):
        Slabs(0.0, 1.0, True, [0.0, 0.6, 0.5, 1.0])


    class OneHoldsAll:
        # four ranks whose particles all sit on this one: the sums over
        # ranks are this rank's own values
        rank, world, tdist = 0, 4, None

        def allreduce(self, value, op, device):
            return float(value)

        def allreduce_tensor(self, t):
            return t

    # balanced cuts give every slab a quarter of a peaked distribution (to
    # within the count of one histogram bin)
    g = torch.from_numpy(np.clip(rng.normal(0.1, 0.15, 10000), -0.5, 0.5))
    s4 = Slabs.balanced(g, -0.5, 0.5, True, OneHoldsAll(), bins=4096)
    shares = np.bincount(s4.owner(g).numpy(), minlength=4)
    assert s4.world == 4 and np.all(np.abs(shares - 2500) < 25), shares
