"""Diagnostic outputs of the equation groups against the oracle.

The reference writes, besides the evolved state, outputs that no later
equation reads: the density pass's rho_sum, arho, grhox/y/z and dwdh
(``src/equations.py:24-86``), the 24 Cullen-Dehnen moments cd_*, the limiter
xilimiter and divvdt (``:283-429``) and StrainDiagnostics' dvdx_*
(``:432-471``).  A ``ParticleArray(diagnostics=True)`` hands these arrays to
the kernels, which then write each one with the reference's semantics; the
checks here compare every one of them with the oracle after the warm-up and
after two PEC steps, on seeded jittered cases (FP64 tolerance 1e-8 relative
to the field's scale, no fallback), and check that writing them leaves the
evolved state unchanged (to FP64 rounding).  Without diagnostics the density passes skip
particles that have converged, so their rho_sum is the sum of the pass in
which they converged (h before the finalisation); the last check bounds that
difference.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import small_cases as sc_  # noqa: E402
from compare import assert_close, scales  # noqa: E402

pytestmark = pytest.mark.gpu

CD = tuple(f"cd_r{a}" for a in ("xx", "xy", "xz", "yy", "yz", "zz")) + tuple(
    f"cd_{q}{a}{b}" for q in "va" for a in "xyz" for b in "xyz")
DVDX = tuple(f"dvdx_{a}{b}" for a in "xyz" for b in "xyz")
DIAG = CD + DVDX + ("xilimiter", "divvdt", "arho", "grhox", "grhoy", "grhoz", "dwdh", "rho_sum")
STATE = ("x", "y", "z", "u", "v", "w", "e", "h", "rho", "p", "cs", "Bx", "By", "Bz", "psi", "alpha1", "au", "av",
         "aw", "ae", "ah", "aBevolx", "aBevoly", "aBevolz", "apsi", "dt_adapt", "alphaloc", "divBsymm", "omega",
         "converged")

CASES = {
    "blast3d_cubic": lambda: sc_.blast_3d(12, "cubic"),
    "blast3d_quintic": lambda: sc_.blast_3d(10, "quintic", hfact=1.0),
    "ot2d_quintic": lambda: sc_.orszag_tang_2d(32, "quintic"),
    "open2d_wendland_c2": lambda: sc_.open_blob_2d(20),
}


def _gpu(ic, prm, steps, diagnostics):
    from src.engine import Engine, params_from_dict
    from src.particle_array import ParticleArray

    eng = Engine(params_from_dict(prm), ParticleArray("fluid", dict(ic), diagnostics=diagnostics))
    eng.warmup()
    out = [eng.pa.pull(*DIAG, *STATE, "gid", order="gid")]
    t, dt = 0.0, eng.initial_dt()
    for _ in range(steps):
        eng.step(dt)
        out.append(eng.pa.pull(*DIAG, *STATE, "gid", order="gid"))
        t += dt
        dt = eng.timestep(t)
    eng.close()
    return out


def _oracle(ic, prm, steps):
    s = oracle.State(dict(ic))
    o = oracle.Oracle(prm, exact_order=False)
    o.warmup(s)
    out = [{k: s[k].copy() for k in DIAG + STATE}]
    t, dt = 0.0, o.initial_dt(s)
    for _ in range(steps):
        o.step(s, dt)
        out.append({k: s[k].copy() for k in DIAG + STATE})
        t += dt
        dt = o.min_dt(s)
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_diagnostic_outputs_match_oracle(name):
    ic, prm = CASES[name]()
    got = _gpu(ic, prm, 2, True)
    ref = _oracle(ic, prm, 2)
    names = DIAG
    for k, (g, r) in enumerate(zip(got, ref)):
        sc = scales(ic, r["cs"])
        assert_close(g, r, names, 1e-8, sc, None, f"{name} {'warm-up' if k == 0 else f'step {k}'} diagnostics")


@pytest.mark.parametrize("name", ("blast3d_cubic", "ot2d_quintic"))
def test_diagnostics_leave_the_state_unchanged(name):
    ic, prm = CASES[name]()
    on = _gpu(ic, prm, 2, True)
    off = _gpu(ic, prm, 2, False)
    for a, b in zip(on, off):
        # the same arithmetic in two kernels; the compiler may contract a
        # multiply-add differently in each, so equal to FP64 rounding
        for k in STATE:
            scale = max(float(np.max(np.abs(a[k]))), 1e-300)
            assert float(np.max(np.abs(a[k] - b[k]))) <= 1e-12 * scale, k
        # rho_sum of a particle that converged before the last pass is the sum
        # of its converging pass (h within the 1e-4 density tolerance of the
        # final one) instead of the last pass's
        rel = np.abs(a["rho_sum"] - b["rho_sum"]) / np.abs(a["rho"])
        assert float(np.max(rel)) <= 1e-3
