"""Neighbour lists carried across sorts.

A list is carried to its particle's new place (renumbered through the sort)
while no pair it lacks can have come within range since it was built, and
rebuilt otherwise.  Checked here: the carried lists still hold every
neighbour under the exact FP64 rule (brute force, after carrying sorts
between steps, on cases with a resting region where lists are carried and a
moving one where they are rebuilt); a run with carried lists equals a run
that rebuilds every list, to FP64 rounding; and a state changed behind the
lists' back (the particle order shuffled between steps) is caught and its
lists rebuilt.
"""

import math
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from test_gpu_neighbours import brute_counts  # noqa: E402

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "u", "v", "w", "rho", "h", "e", "Bx", "By", "Bz", "psi", "alpha1")


def blast_lattice(n=18, radius=0.2):
    """The 3-D blast on an unjittered lattice: outside the hot sphere the gas
    rests until the wave arrives, so its lists are carried over."""
    dx = 1.0 / n
    ax = -0.5 + (np.arange(n) + 0.5) * dx
    x, y, z = (a.ravel() for a in np.meshgrid(ax, ax, ax, indexing="ij"))
    cnt = x.size
    gamma = 5.0 / 3.0
    p = np.where(x * x + y * y + z * z < radius * radius, 10.0, 0.1)
    b = 1.0 / math.sqrt(2.0)
    ic = dict(x=x, y=y, z=z, u=np.zeros(cnt), v=np.zeros(cnt), w=np.zeros(cnt), rho=np.ones(cnt),
              h=np.full(cnt, 1.2 * dx), m=np.full(cnt, dx ** 3), e=p / (gamma - 1.0), Bx=np.full(cnt, b),
              By=np.full(cnt, b), Bz=np.zeros(cnt), alpha1=np.full(cnt, 0.1), gid=np.arange(cnt, dtype=np.float64))
    prm = dict(dim=3, kernel="cubic", hfact=1.2, density="iterate", gamma=gamma, mu0=1.0, av=1.0, ac=1.0, ar=1.0,
               clean_speed=1.0, clean_damp=1.0, timestep_factor=1.0, tf=1e30, lo=[-0.5] * 3, hi=[0.5] * 3,
               periodic=[True] * 3, alpha_min=0.1, alpha_max=1.0)
    return ic, prm


def shock_tube(nx=96):
    """The 2-D Brio-Wu tube of configs/mhdshock2d.toml at a smaller nx: the
    ends rest (and are frozen) while the waves run from the middle."""
    from dataclasses import replace

    from src.config import load_config
    from src.run import CASES

    root = os.path.join(os.path.dirname(__file__), "..", "pysph-mhd_b200", "configs", "mhdshock2d.toml")
    cfg = load_config(root, {k: v.config_type for k, v in CASES.items()})
    cfg = replace(cfg, case=replace(cfg.case, nx=nx))
    app = CASES[cfg.case.name](cfg)
    ic = app.create_mhd_particles()
    prm = app.scheme.kernel_params(app.create_domain(), app.tf)
    return ic, dict(prm, precision="fp64")


# small enough for the brute-force check, large enough that a resting region
# outlives the dilation of the moving one by the stencil for a few steps
CASES = {"blast_lattice_3d": blast_lattice, "shock_tube_2d": shock_tube}
# over 20 steps
LONG_CASES = {"blast_lattice_3d": lambda: blast_lattice(32, 0.1), "shock_tube_2d": lambda: shock_tube(128)}


def _engine(ic, prm):
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray

    return Engine(params_from_dict(prm), ParticleArray("fluid", dict(ic)))


def _list_counts(eng):
    import ctypes

    listed, rebuilt = ctypes.c_int64(), ctypes.c_int64()
    eng._check(eng.lib.mhd_list_counts(eng.ctx, ctypes.byref(listed), ctypes.byref(rebuilt), eng.stream))
    return listed.value, rebuilt.value


def _check_counts(eng, prm, what):
    counts = eng.neighbour_counts().cpu().numpy()
    st = eng.pa.pull("x", "y", "z", "h")
    ref = brute_counts(st["x"], st["y"], st["z"], st["h"], prm)
    bad = np.nonzero(counts != ref)[0]
    assert bad.size == 0, f"{what}: {bad.size} particles differ, e.g. {bad[:5]}: {counts[bad[:5]]} vs {ref[bad[:5]]}"


@pytest.mark.parametrize("name", sorted(CASES))
def test_carried_lists_hold_exact_neighbour_sets(name):
    ic, prm = CASES[name]()
    eng = _engine(ic, prm)
    eng.warmup()
    eng.begin(eng.initial_dt())
    _list_counts(eng)
    carried = 0
    for k in range(8):
        eng.advance(1, finish=False)
        if k % 2 == 1:
            # the lists of the last right-hand side were built before the
            # corrector-predictor moved the particles: sort again (carrying
            # them) and check the lists of the current positions
            eng.cells_build()
            _check_counts(eng, prm, f"{name} after fused step {k + 1}")
        listed, rebuilt = _list_counts(eng)
        carried += listed - rebuilt
    eng.close()
    assert carried > 0, "no list was carried over: the test does not exercise the carry"


@pytest.mark.parametrize("name", sorted(LONG_CASES))
def test_carried_lists_match_full_rebuilds(name, monkeypatch):
    ic, prm = LONG_CASES[name]()
    out, stats = {}, {}
    for reuse in ("1", "0"):
        monkeypatch.setenv("MHD_LIST_REUSE", reuse)
        eng = _engine(ic, prm)
        eng.warmup()
        eng.begin(eng.initial_dt())
        _list_counts(eng)
        eng.advance(20)
        stats[reuse] = _list_counts(eng)
        out[reuse] = eng.pa.pull(*FIELDS, "gid", order="gid")
        eng.close()
    assert stats["0"][1] == stats["0"][0]  # every list rebuilt
    assert stats["1"][1] < stats["1"][0]
    for f in FIELDS:
        a, b = out["1"][f], out["0"][f]
        scale = max(np.linalg.norm(b), 1e-300)
        err = np.linalg.norm(a - b) / scale
        assert err <= 1e-11, f"{name} {f}: carried vs rebuilt lists differ by {err:.3e}"


def test_shuffled_state_is_caught():
    # after a few steps, permute the particles of the current state: the
    # carried lists name the old order; the displacement test must see the
    # mismatch and rebuild what the shuffle touched
    ic, prm = blast_lattice(24, 0.12)
    eng = _engine(ic, prm)
    eng.warmup()
    eng.begin(eng.initial_dt())
    eng.advance(3, finish=False)
    n = eng.pa.n
    # shuffle a window of 300 consecutive slots near the start of the sorted
    # order (a resting corner of the box): most lists are still carried, the
    # ones naming the window must not be
    g = torch.Generator(device="cpu").manual_seed(7)
    win = torch.arange(n)
    lo = 40
    win[lo:lo + 300] = lo + torch.randperm(300, generator=g)
    win = win.to(eng.pa.device)
    for k, v in eng.pa.properties.items():
        v.copy_(v[win])
    _list_counts(eng)
    eng.cells_build()
    listed, rebuilt = _list_counts(eng)
    assert 0 < rebuilt < listed
    _check_counts(eng, prm, "after a shuffle of the state")
    eng.close()
