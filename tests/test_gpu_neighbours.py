"""Neighbour sets of the compacted lists, exact against brute force.

The neighbour rule (PySPH's NNPS, restated): j is a neighbour of i when
r2 < (R h_i)^2 or r2 < (R h_j)^2, with r2 = (dx dx + dy dy) + dz dz on the
minimum-image displacement, self included.  The device counts neighbours
with that FP64 rule over each particle's list; brute force over all pairs on
the host must give identical counts -- for the initial state, and after a
density iteration has changed h.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import small_cases as sc_  # noqa: E402
from golden_io import CASES, load, section  # noqa: E402

pytestmark = pytest.mark.gpu

R = {"cubic": 2.0, "quintic": 3.0, "wendland_c2": 2.0, "wendland_c4": 2.0, "wendland_c6": 2.0, "gaussian": 3.0,
     "super_gaussian": 3.0}


def brute_counts(x, y, z, h, prm):
    lo, hi, per = prm["lo"], prm["hi"], prm["periodic"]
    pos = [x, y, z]
    n = len(x)
    rh = R[prm["kernel"]] * h
    rh2 = rh * rh
    out = np.zeros(n, dtype=np.int64)
    for i in range(n):
        d = []
        for a in range(3):
            if a >= prm["dim"]:
                d.append(np.zeros(n))
                continue
            v = pos[a][i] - pos[a]
            if per[a]:
                L = hi[a] - lo[a]
                half = 0.5 * L
                v = np.where(v > half, v - L, v)
                v = np.where(v < -half, v + L, v)
            d.append(v)
        r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
        out[i] = int(np.count_nonzero((r2 < rh2[i]) | (r2 < rh2)))
    return out


def _engine(ic, prm):
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray

    return Engine(params_from_dict(prm), ParticleArray("fluid", ic))


def _check(eng, prm, what):
    counts = eng.neighbour_counts().cpu().numpy()
    st = eng.pa.pull("x", "y", "z", "h")
    ref = brute_counts(st["x"], st["y"], st["z"], st["h"], prm)
    bad = np.nonzero(counts != ref)[0]
    assert bad.size == 0, f"{what}: {bad.size} particles differ, e.g. {bad[:5]}: {counts[bad[:5]]} vs {ref[bad[:5]]}"


@pytest.mark.parametrize("case", CASES)
def test_lists_hold_exact_neighbour_sets_golden(case):
    d, p = load(case)
    eng = _engine(section(d, "ic"), p)
    eng.cells_build()
    _check(eng, p, f"{case} initial")
    eng.warmup()  # three RHS: density iterations move h, lists are rebuilt
    eng.cells_build()
    _check(eng, p, f"{case} after warm-up")


@pytest.mark.parametrize("maker", [lambda: sc_.orszag_tang_2d(32, "quintic"), lambda: sc_.blast_3d(12, "cubic"),
                                   lambda: sc_.open_blob_2d(20)])
def test_lists_hold_exact_neighbour_sets_jittered(maker):
    ic, prm = maker()
    eng = _engine(ic, prm)
    eng.warmup()
    eng.cells_build()
    _check(eng, prm, "jittered after warm-up")


def _spread_h(ic, frac, factors, seed):
    """A few particles get a much larger h: they become the grid's big
    particles, whose pairs come from the extended search and the scatter."""
    rng = np.random.default_rng(seed)
    ic = dict(ic)
    h = ic["h"].copy()
    pick = rng.random(h.size) < frac
    h[pick] *= rng.choice(factors, pick.sum())
    ic["h"] = h
    return ic


@pytest.mark.parametrize("maker,frac", [(lambda: sc_.orszag_tang_2d(40, "quintic"), 0.03),
                                        (lambda: sc_.blast_3d(14, "cubic"), 0.02),
                                        (lambda: sc_.open_blob_2d(30), 0.05),
                                        (lambda: sc_.blast_3d(12, "cubic"), 0.3)])
def test_lists_exact_with_a_few_large_h(maker, frac):
    ic, prm = maker()
    ic = _spread_h(ic, frac, [1.3, 2.0, 3.5], seed=4)
    eng = _engine(ic, prm)
    eng.cells_build()
    _check(eng, prm, f"large h (fraction {frac})")


@pytest.mark.parametrize("maker", [lambda: sc_.orszag_tang_2d(36, "quintic"), lambda: sc_.blast_3d(12, "cubic"),
                                   lambda: sc_.open_blob_2d(24)])
@pytest.mark.parametrize("spread", [0.15, 0.6])
def test_lists_exact_with_continuously_spread_h(maker, spread):
    # h spread continuously: many particles fall between the h the cells follow
    # and the largest h their stencil covers, others become big
    ic, prm = maker()
    rng = np.random.default_rng(int(spread * 100))
    ic = dict(ic, h=ic["h"] * (1.0 + spread * rng.random(ic["h"].size)))
    eng = _engine(ic, prm)
    eng.cells_build()
    _check(eng, prm, f"continuous h spread {spread}")


def test_lists_exact_through_steps_open_blob():
    # an expanding open blob: h grows at its rim from step to step
    ic, prm = sc_.open_blob_2d(20)
    eng = _engine(ic, prm)
    eng.warmup()
    dt, t = eng.initial_dt(), 0.0
    for _ in range(4):
        eng.step(dt)
        t += dt
        dt = eng.timestep(t)
        _check(eng, prm, "open blob after a step")


def test_batched_lists_exact_with_a_few_large_h():
    from src.batch import BatchEngine
    from src.engine import params_from_dict

    a, prm = sc_.orszag_tang_2d(24, "quintic", seed=1)
    b, _ = sc_.orszag_tang_2d(33, "quintic", seed=2)
    ics = [_spread_h(a, 0.04, [2.0, 3.0], 5), _spread_h(b, 0.02, [1.5, 2.5], 6)]
    eng = BatchEngine(params_from_dict(prm), ics)
    eng.cells_build()
    counts = eng.neighbour_counts().cpu().numpy()
    for k in range(2):
        sl = eng.instance(k)
        st = {f: eng.pa[f][sl].cpu().numpy() for f in ("x", "y", "z", "h")}
        ref = brute_counts(st["x"], st["y"], st["z"], st["h"], prm)
        bad = np.nonzero(counts[sl] != ref)[0]
        assert bad.size == 0, f"instance {k}: {bad.size} particles differ"
    eng.close()


def test_long_appended_runs_are_ordered_deterministically():
    # A blob of large-h particles: each smaller particle near it gets dozens
    # of entries scattered into its list (runs longer than a warp), which the
    # ordering pass must put in index order whatever order the scatter's
    # atomics left them in.  The lists hold the exact neighbour sets, and two
    # warm-ups (three right-hand sides each) from the same state agree bit for
    # bit.
    ic, prm = sc_.blast_3d(16, "cubic")
    r2 = ic["x"] ** 2 + ic["y"] ** 2 + ic["z"] ** 2
    ic = dict(ic, h=np.where(r2 < 0.18 ** 2, 3.0, 1.0) * ic["h"])
    outs = []
    for _ in range(2):
        eng = _engine(ic, prm)
        eng.cells_build()
        _check(eng, prm, "large-h blob")
        eng.warmup()
        outs.append(eng.pa.pull("au", "av", "aw", "ae", "aBevolx", "rho", "h", "gid", order="gid"))
        eng.close()
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), f"{k} differs between two identical runs"
