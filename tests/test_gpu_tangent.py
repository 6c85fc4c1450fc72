"""Derivative form (forward mode) of the SPMHD step.

* Its primal values are the FP64 drop-in path's (single density pass,
  literal PEC steps with the same step sizes), to roundoff.
* Its derivatives match central finite differences of the FP64 drop-in
  path with the step sizes frozen, for the final magnetic energy of the
  Alfven wave (amplitude and alpha_max) and for an arbitrary seed direction
  of a 3-D case.
"""

import os
from dataclasses import replace

import numpy as np
import pytest

pytest.importorskip("torch")

import small_cases as sc_  # noqa: E402
from compare import assert_close, scales  # noqa: E402

pytestmark = pytest.mark.gpu

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pysph-mhd_b200")
FIELDS = ("x", "y", "u", "v", "w", "rho", "h", "e", "Bx", "By", "Bz", "alpha1", "au", "av", "ae", "psi")


def _alfven_config(nx):
    from src.config import load_config
    from src.run import CASES

    cfg = load_config(os.path.join(PKG, "configs", "alfven2d.toml"), {k: v.config_type for k, v in CASES.items()})
    return replace(cfg, case=replace(cfg.case, nx=nx))


def _production(ic, prm, dts):
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray

    eng = Engine(params_from_dict(dict(prm, density="single")), ParticleArray("fluid", dict(ic)))
    eng.warmup()
    for dt in dts:
        eng.step(dt)
    out = eng.pa.pull(*FIELDS, "m", "gid", order="gid")
    eng.close()
    return out


def _tangent(ic, prm, steps, dts=None, seeds=None, amax_seed=None):
    from src.derivative import TangentEngine, TangentState
    from src.engine import params_from_dict

    eng = TangentEngine(params_from_dict(dict(prm, density="single")), TangentState(dict(ic), seeds),
                        alpha_max_seed=amax_seed)
    eng.warmup()
    eng.run(steps, dts)
    return eng


def _energy(out, mu0=1.0):
    b2 = out["Bx"] ** 2 + out["By"] ** 2 + out["Bz"] ** 2
    return float(np.sum(out["m"] * b2 / (2.0 * mu0 * out["rho"])))


@pytest.mark.parametrize("name", ["ot2d", "blast3d", "alfven"])
def test_primal_values_match_the_drop_in_path(name):
    if name == "alfven":
        from src.derivative import alfven_case

        ic, _, prm = alfven_case(_alfven_config(16), 0.1, 1.0)
    elif name == "ot2d":
        ic, prm = sc_.orszag_tang_2d(20, "quintic", seed=4)
    else:
        ic, prm = sc_.blast_3d(8, "cubic", seed=6)
    eng = _tangent(ic, prm, 4)
    got = {k: eng.ts.value(k).cpu().numpy() for k in FIELDS}
    dts = list(eng.dts)
    eng.close()
    ref = _production(ic, prm, dts)
    assert_close(got, ref, FIELDS, 1e-10, scales(ic, ref["rho"] * 0 + 1.0), None, f"{name} tangent primal")


def test_alfven_gradient_matches_central_differences():
    from src.derivative import alfven_case, magnetic_energy_and_gradient

    cfg = _alfven_config(16)
    amp, amax, steps = 0.1, 1.0, 12
    value, grad, dts = magnetic_energy_and_gradient(cfg, amp, amax, steps)

    def loss(a, am):
        ic, _, prm = alfven_case(cfg, a, am)
        return _energy(_production(ic, prm, dts))

    assert abs(loss(amp, amax) - value) <= 1e-11 * abs(value)
    ea = 1e-5 * amp
    fd_a = (loss(amp + ea, amax) - loss(amp - ea, amax)) / (2 * ea)
    assert abs(grad[0] - fd_a) <= 1e-6 * abs(fd_a), (grad[0], fd_a)
    # A linear Alfven wave does not compress: alpha_loc stays ~1e-8, far below
    # alpha_max, so the clip is inactive and the loss does not depend on it.
    assert grad[1] == 0.0
    assert loss(amp, amax + 0.1) == loss(amp, amax - 0.1)


def test_alpha_max_gradient_on_a_blast_matches_central_differences():
    # the blast's shock drives alpha_loc to the clip, so alpha_max matters
    ic, prm = sc_.blast_3d(8, "cubic", seed=3, alpha=(0.1, 0.6))
    eng = _tangent(ic, prm, 6, seeds={"e": [0.01 * ic["e"], None]}, amax_seed=[0.0, 1.0])
    clipped = int((eng.ts.value("alphaloc") == 0.6).sum())
    value, grad = eng.magnetic_energy()
    dts = list(eng.dts)
    eng.close()
    assert clipped > 0

    def loss(scale_e, am):
        return _energy(_production(dict(ic, e=ic["e"] * (1.0 + 0.01 * scale_e)), dict(prm, alpha_max=am), dts))

    assert abs(loss(0.0, 0.6) - value) <= 1e-11 * abs(value)
    h = 1e-6
    fd_e = (loss(h, 0.6) - loss(-h, 0.6)) / (2 * h)
    fd_m = (loss(0.0, 0.6 + h) - loss(0.0, 0.6 - h)) / (2 * h)
    assert grad[1] != 0.0
    assert abs(grad[0] - fd_e) <= 1e-5 * abs(fd_e), (grad[0], fd_e)
    assert abs(grad[1] - fd_m) <= 1e-4 * abs(fd_m), (grad[1], fd_m)


def test_seeded_direction_matches_central_differences_3d():
    # d(magnetic energy)/d(theta) for x(theta) = x0 + theta * dx, e(theta) = e0 + theta * de
    ic, prm = sc_.blast_3d(8, "cubic", seed=9)
    rng = np.random.default_rng(1)
    dx = 0.05 / 8 * rng.uniform(-1, 1, ic["x"].size)
    de = 0.1 * ic["e"] * rng.uniform(-1, 1, ic["e"].size)
    eng = _tangent(ic, prm, 5, seeds={"x": [dx, None], "e": [None, de]})
    value, grad = eng.magnetic_energy()
    dts = list(eng.dts)
    eng.close()

    def loss(th_x, th_e):
        ic2 = dict(ic, x=ic["x"] + th_x * dx, e=ic["e"] + th_e * de)
        return _energy(_production(ic2, prm, dts))

    assert abs(loss(0.0, 0.0) - value) <= 1e-11 * abs(value)
    h = 1e-5
    fd_x = (loss(h, 0.0) - loss(-h, 0.0)) / (2 * h)
    fd_e = (loss(0.0, h) - loss(0.0, -h)) / (2 * h)
    assert abs(grad[0] - fd_x) <= 1e-5 * max(abs(fd_x), 1e-12 * abs(value)), (grad[0], fd_x)
    assert abs(grad[1] - fd_e) <= 1e-5 * max(abs(fd_e), 1e-12 * abs(value)), (grad[1], fd_e)
