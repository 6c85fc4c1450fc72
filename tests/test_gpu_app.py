"""The reference-facing path end to end: TOML -> case -> MHDApplication.run().

``src.run.main`` mirrors ``python -m src.run <config>`` (src/run.py:32-39):
the application warms up, takes the initial dt and runs MHDSolver.solve with
the fused loop (``execution.fused``) or the literal PEC step; the result must
match the oracle driven the same way.
"""

import os

import numpy as np
import pytest

pytest.importorskip("torch")

import oracle  # noqa: E402
from compare import assert_close, scales  # noqa: E402

pytestmark = pytest.mark.gpu

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pysph-mhd_b200")


def _small_config(tmp_path, name, nx, steps, extra=""):
    text = open(os.path.join(PKG, "configs", f"{name}.toml")).read()
    text = text.replace("max_steps = 100", f"max_steps = {steps}").replace("max_steps = 50", f"max_steps = {steps}")
    import re

    text = re.sub(r"nx = \d+", f"nx = {nx}", text)
    text = text.replace('directory = "outputs/', f'directory = "{tmp_path}/')
    p = tmp_path / f"{name}.toml"
    p.write_text(text + extra)
    return str(p)


@pytest.mark.parametrize("fused", [True, False])
def test_run_blast3d_config_matches_oracle(tmp_path, fused):
    # execution.fused: captured chunks of corrector-predictor steps with the
    # step size on the device; otherwise the literal MHDStep stages
    from src.run import main

    path = _small_config(tmp_path, "mhdblast3d", 12, 3)
    text = open(path).read().replace('precision = "fp32"', 'precision = "fp64"')
    if not fused:
        text = text.replace("fused = true", "fused = false")
    open(path, "w").write(text)
    app, pa = main([path])
    assert app.solver.fused is fused
    got = pa.pull("x", "u", "v", "rho", "e", "Bx", "By", "alpha1", "h", order="gid")
    assert app.solver.count == 3

    ic = app.create_mhd_particles()
    ic["gid"] = np.arange(len(ic["x"]), dtype=float)
    prm = app.scheme.kernel_params(app.create_domain(), app.tf)
    s = oracle.State(ic)
    o = oracle.Oracle(prm, exact_order=False)
    o.warmup(s)
    o.run(s, 3, tf=app.tf)
    ref = {k: s[k] for k in got if k != "gid"}
    assert_close(got, ref, list(ref), 1e-8, scales(ic, s["cs"]), None, "src.run mhdblast3d")
    # output dumps: initial, final
    dumps = sorted(os.listdir(os.path.join(tmp_path, "mhdblast3d")))
    assert dumps[0].endswith("000000.npz") and dumps[-1].endswith("000003.npz")


def test_restart_from_detailed_dump_continues_the_run(tmp_path):
    # run 4 steps dumping every property every 2 steps; a second application
    # restarted from the step-2 dump must reach the same step-4 state
    import re

    from src.config import load_config
    from src.run import CASES

    path = _small_config(tmp_path, "mhdblast3d", 10, 4)
    text = open(path).read().replace('precision = "fp32"', 'precision = "fp64"')
    text = re.sub(r"pfreq = \d+", "pfreq = 2", text)
    open(path, "w").write(text)
    types = {k: v.config_type for k, v in CASES.items()}

    app = CASES["mhdblast3d"](load_config(path, types))
    app.detailed_output = True
    full = app.run().pull("x", "y", "u", "v", "rho", "e", "Bx", "By", "psi", "alpha1", "h", order="gid")
    assert app.solver.count == 4
    dump = os.path.join(tmp_path, "mhdblast3d", "mhdblast3d_000002.npz")

    app2 = CASES["mhdblast3d"](load_config(path, types))
    app2.detailed_output = True
    again = app2.restart(dump).pull(*full, order="gid")
    assert app2.solver.count == 4
    for k in full:
        scale = max(float(np.max(np.abs(full[k]))), 1e-300)
        assert float(np.max(np.abs(again[k] - full[k]))) <= 1e-10 * scale, k
