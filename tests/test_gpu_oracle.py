"""CUDA path against the C oracle on well-conditioned seeded cases.

Covers every kernel of the reference's kernel map (src/scheme.py:48-56),
dim 2 and 3, periodic and open boundaries (periodic_mode None), the
alpha_min/alpha_max extension and both the literal PEC step and the fused
corrector-predictor loop.  Tolerances: FP64 rounding only.
"""

import numpy as np
import pytest

pytest.importorskip("torch")

import oracle  # noqa: E402
import small_cases as sc_  # noqa: E402
from compare import assert_close, scales  # noqa: E402

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "u", "v", "w", "e", "h", "rho", "p", "cs", "Bx", "By", "Bz", "psi", "alpha1", "au",
          "av", "aw", "ae", "ah", "aBevolx", "aBevoly", "aBevolz", "apsi", "dt_adapt", "alphaloc", "divBsymm",
          "omega")


def _run_gpu(ic, prm, steps, fused=False):
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray

    eng = Engine(params_from_dict(prm), ParticleArray("fluid", ic))
    eng.warmup()
    dt0 = eng.initial_dt()
    dts = []
    if fused:
        eng.begin(dt0)
        eng.advance(steps)
    else:
        t, dt = 0.0, dt0
        for _ in range(steps):
            dts.append(dt)
            eng.step(dt)
            t += dt
            dt = eng.timestep(t)
    out = eng.pa.pull(*FIELDS, "gid", order="gid")
    eng.close()
    return out, dt0, dts


def _run_oracle(ic, prm, steps):
    s = oracle.State(ic)
    o = oracle.Oracle(prm, exact_order=False)
    o.warmup(s)
    dt0 = o.initial_dt(s)
    rec = o.run(s, steps, tf=prm["tf"])
    return {k: s[k] for k in FIELDS}, dt0, [r[1] for r in rec]


CASES = {
    "ot2d_quintic": lambda: sc_.orszag_tang_2d(32, "quintic"),
    "ot2d_cubic": lambda: sc_.orszag_tang_2d(32, "cubic", hfact=1.3),
    "ot2d_wendland_c4": lambda: sc_.orszag_tang_2d(24, "wendland_c4", hfact=1.4),
    "ot2d_gaussian": lambda: sc_.orszag_tang_2d(24, "gaussian", hfact=1.0),
    "blast3d_cubic_alpha01": lambda: sc_.blast_3d(12, "cubic"),
    "blast3d_wendland_c6": lambda: sc_.blast_3d(10, "wendland_c6", hfact=1.5),
    "blast3d_quintic": lambda: sc_.blast_3d(10, "quintic", hfact=1.0),
    "blast3d_super_gaussian": lambda: sc_.blast_3d(10, "super_gaussian", hfact=1.0),
    "open2d_wendland_c2": lambda: sc_.open_blob_2d(20),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_pec_steps_match_oracle(name):
    ic, prm = CASES[name]()
    got, dt0, dts = _run_gpu(ic, prm, 4)
    ref, dt0_ref, dts_ref = _run_oracle(ic, prm, 4)
    assert abs(dt0 - dt0_ref) <= 1e-10 * dt0_ref
    np.testing.assert_allclose(dts, dts_ref, rtol=1e-8)
    assert_close(got, ref, FIELDS, 1e-8, scales(ic, ref["cs"]), None, name)


@pytest.mark.parametrize("name", ("ot2d_quintic", "blast3d_cubic_alpha01", "open2d_wendland_c2"))
def test_fused_loop_matches_oracle(name):
    ic, prm = CASES[name]()
    got, _, _ = _run_gpu(ic, prm, 4, fused=True)
    ref, _, _ = _run_oracle(ic, prm, 4)
    assert_close(got, ref, FIELDS, 1e-8, scales(ic, ref["cs"]), None, name + " fused")


def test_density_single_pass_mode():
    """numerics.density = "single": one pass, every particle finalised."""
    ic, prm = sc_.orszag_tang_2d(24, "quintic")
    prm = dict(prm, density="single")
    got, _, _ = _run_gpu(ic, prm, 2)
    ref, _, _ = _run_oracle(ic, prm, 2)
    assert_close(got, ref, FIELDS, 1e-8, scales(ic, ref["cs"]), None, "single")
