"""The reference's other case generators on the CUDA path.

Each case (sine, magnetosonic pulse, rotor, advected vortex, current loop,
one/three/twelve colliding jets) is built from its TOML file at a small nx by
the package's generators (checked against the reference's own output on the
CPU, tests/test_app_cpu.py), then warmed up and advanced two PEC steps on the
GPU and by the C oracle.  The cases bring in what the benchmark
configurations do not: Wendland C4/C6 at large hfact, open boundaries with
SI-unit magnitudes (the jets), a two-spacing lattice (the rotor), zero
dissipation.  Tolerance: FP64 rounding only.
"""

import os
from dataclasses import replace

import numpy as np
import pytest

pytest.importorskip("torch")

import oracle  # noqa: E402
from compare import assert_close, scales  # noqa: E402

pytestmark = pytest.mark.gpu

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pysph-mhd_b200")
FIELDS = ("x", "y", "z", "u", "v", "w", "e", "h", "rho", "p", "cs", "Bx", "By", "Bz", "psi", "au", "av", "aw", "ae",
          "aBevolx", "aBevoly", "aBevolz", "apsi", "dt_adapt", "divBsymm", "omega")
SIZES = {"mhdsine": 12, "mhdwave": 16, "mhdrotor": 16, "mhdvortex": 12, "jadvect": 12, "1jet": 6, "3jet": 5,
         "12jet": 4}


def _case(name):
    from src.config import load_config
    from src.run import CASES

    cfg = load_config(os.path.join(PKG, "configs", f"{name}.toml"), {k: v.config_type for k, v in CASES.items()})
    cfg = replace(cfg, case=replace(cfg.case, nx=SIZES[name]))
    app = CASES[name](cfg)
    ic = app.create_mhd_particles()
    ic.setdefault("gid", np.arange(len(ic["x"]), dtype=np.float64))
    return ic, app.scheme.kernel_params(app.create_domain(), app.tf)


@pytest.mark.parametrize("name", sorted(SIZES))
def test_case_steps_match_oracle(name):
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray

    ic, prm = _case(name)
    eng = Engine(params_from_dict(prm), ParticleArray("fluid", dict(ic)))
    eng.warmup()
    dt0 = eng.initial_dt()
    t, dt = 0.0, dt0
    for _ in range(2):
        eng.step(dt)
        t += dt
        dt = eng.timestep(t)
    got = eng.pa.pull(*FIELDS, "gid", order="gid")
    eng.close()

    s = oracle.State(ic)
    o = oracle.Oracle(prm, exact_order=False)
    o.warmup(s)
    dt0_ref = o.initial_dt(s)
    o.run(s, 2, tf=prm["tf"])
    ref = {k: s[k] for k in FIELDS}
    assert abs(dt0 - dt0_ref) <= 1e-10 * dt0_ref
    assert_close(got, ref, FIELDS, 1e-8, scales(ic, ref["cs"]), None, name)
