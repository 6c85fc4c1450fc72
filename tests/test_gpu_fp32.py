"""FP32 precision form against the FP64 path (and the oracle).

The FP32 form computes pair arithmetic in single precision with
Kahan-compensated sums and keeps the density Newton iteration, the
epilogues, the integrator and the timestep reduction in FP64.  Its error
against the FP64 run is stated per field as a relative L2 norm.
"""

import numpy as np
import pytest

pytest.importorskip("torch")

import small_cases as sc_  # noqa: E402

pytestmark = pytest.mark.gpu

FIELDS = ("rho", "u", "v", "w", "Bx", "By", "Bz", "e", "h", "psi", "alpha1")


def _run(ic, prm, precision, steps):
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray

    eng = Engine(params_from_dict(prm, precision), ParticleArray("fluid", ic))
    eng.warmup()
    eng.begin(eng.initial_dt())
    eng.advance(steps)
    out = eng.pa.pull(*FIELDS, "gid", order="gid")
    eng.close()
    return out


def _rel_l2(a, b):
    den = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / den if den > 0 else float(np.linalg.norm(a - b))


@pytest.mark.parametrize("name,steps", [("ot2d", 10), ("blast3d", 10), ("blast3d_quintic", 6)])
def test_fp32_form_close_to_fp64(name, steps):
    ic, prm = {"ot2d": lambda: sc_.orszag_tang_2d(32, "quintic"),
               "blast3d": lambda: sc_.blast_3d(12, "cubic"),
               "blast3d_quintic": lambda: sc_.blast_3d(10, "quintic", hfact=1.0)}[name]()
    ref = _run(ic, prm, "fp64", steps)
    got = _run(ic, prm, "fp32", steps)
    errs = {k: _rel_l2(got[k], ref[k]) for k in FIELDS if np.any(ref[k])}
    for k in ("rho", "u", "v", "Bx", "By"):
        assert errs[k] < 1e-5, f"{name} FP32 vs FP64 rel L2 {k} = {errs[k]:.2e} ({errs})"
    assert max(errs.values()) < 1e-4, errs


@pytest.mark.parametrize("name", ["blast3d", "ot2d"])
def test_cell_tile_force_pass_equals_list_pass(name, monkeypatch):
    # The cell-tile force pass (MHD_FORCE_TILES=1, kept for comparison with
    # the list-driven pass) visits the same pairs -- no particle is big in
    # these warm-ups, whose h stays uniform -- in another order: FP32 sums
    # agree to a few rounding errors of the pair terms.
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray

    ic, prm = {"blast3d": lambda: sc_.blast_3d(16, "cubic"), "ot2d": lambda: sc_.orszag_tang_2d(40, "quintic")}[name]()
    names = ("au", "av", "ae", "aBevolx", "aBevoly", "apsi", "dt_adapt", "alphaloc", "divBsymm")
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("MHD_FORCE_TILES", mode)
        eng = Engine(params_from_dict(prm, "fp32"), ParticleArray("fluid", ic))
        eng.warmup()
        out[mode] = eng.pa.pull(*names, order="gid")
        eng.close()
    for k in names:
        ref = out["0"][k]
        err = float(np.max(np.abs(out["1"][k] - ref))) / max(float(np.max(np.abs(ref))), 1e-300)
        assert err < 2e-5, (k, err)
