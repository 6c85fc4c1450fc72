"""The C oracle against fixtures made by executing the reference's own code.

The fixtures (``tests/golden/make_golden.py``) run the reference's
``src/equations.py``, ``src/integrator.py``, ``MHDScheme.get_equations``,
``MHDApplication._warm_initial_derivatives`` / ``_compute_initial_dt`` and
``MHDSolver.solve`` in pure Python.  With neighbours summed in ascending
index order the oracle must reproduce them bit for bit.
"""

import numpy as np
import pytest

import oracle
from golden_io import CASES, load, section

WARM_FIELDS = ("rho", "h", "omega", "cs", "p", "au", "av", "aw", "ae", "ah", "dt_cfl", "dt_adapt", "alphaloc",
               "aBevolx", "aBevoly", "aBevolz", "apsi", "Bx", "By", "Bz", "divBsymm", "divBdiff", "div",
               "xilimiter", "divvdt", "converged", "rho_sum")
STEP_FIELDS = ("x", "y", "z", "u", "v", "w", "e", "h", "h0", "rho", "p", "cs", "Bx", "By", "Bz", "Bevolx", "Bevoly",
               "Bevolz", "psi", "alpha1", "au", "av", "aw", "ae", "ah", "dt_adapt", "omega")


@pytest.fixture(scope="module", autouse=True)
def _built():
    oracle.build()


@pytest.mark.parametrize("case", CASES)
def test_oracle_bit_exact_against_reference_code(case):
    d, p = load(case)
    s = oracle.State(section(d, "ic"))
    o = oracle.Oracle(p, exact_order=True, nthreads=2)
    o.warmup(s)
    warm = section(d, "warm")
    for k in WARM_FIELDS:
        np.testing.assert_array_equal(s[k], warm[k], err_msg=f"warm-up field {k}")
    dt0 = o.initial_dt(s)
    assert dt0 == float(d["dt0"])
    seen = []

    def cb(k, st, t, dt):
        ref = section(d, f"step{k}")
        for f in STEP_FIELDS:
            np.testing.assert_array_equal(st[f], ref[f], err_msg=f"step {k} field {f}")
        seen.append(dt)

    o.run(s, int(d["n_steps"]), tf=p["tf"], callback=cb)
    np.testing.assert_array_equal(np.array(seen), d["step_dt"])
    assert o.density_passes == list(d["density_passes"])


@pytest.mark.parametrize("case", ("ot2d", "blast3d"))
def test_oracle_cell_order_close_to_exact_order(case):
    """Summation in cell order (the timed CPU baseline) differs only by rounding."""
    d, p = load(case)
    a = oracle.State(section(d, "ic"))
    b = oracle.State(section(d, "ic"))
    oracle.Oracle(p, exact_order=True).warmup(a)
    oracle.Oracle(p, exact_order=False).warmup(b)
    for k in ("rho", "h", "au", "ae", "aBevolx", "dt_adapt"):
        np.testing.assert_allclose(b[k], a[k], rtol=1e-11, atol=1e-11 * np.max(np.abs(a[k])))
