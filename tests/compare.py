"""Field comparison for the parity tests.

Two facts shape the criteria:

* Several fields vanish analytically for the test initial conditions
  (div v for Orszag-Tang's incompressible start, div B for a uniform field),
  so they are pure roundoff; each field is therefore compared relative to
  max(max|ref|, a physical floor built from the case's velocity, field,
  density and smoothing-length scales).
* The reference's Cullen-Dehnen limiter xi = (-div v)^2 / ((div v)^2 +
  |curl v|^2) is roundoff / roundoff where both vanish (Orszag-Tang's
  stagnation lines at t = 0): the reference restated bit-exactly flips
  alpha_loc between 0 and 1 on some particles just by summing neighbours in
  a different order.  Only the fields named in ``ROUNDOFF_SENSITIVE`` (the
  limiter and the switch it drives), plus any a test names explicitly, may
  then lie within the reference's own reordering spread instead:
  ||gpu - ref||_2 <= 10 ||ref' - ref||_2, where ref' is the oracle summed in
  cell order.  With MHD_SPREAD_REPORT set, every use of that fallback is
  appended to the named file as a JSON line.
"""

import json
import os

import numpy as np

FAMILY = {
    "ah": "V", "div": "V/H", "div_for_psi": "V/H", "divBsymm": "B/H", "divBdiff": "RB/H", "apsi": "VB/H",
    "aBevolx": "BV/RH", "aBevoly": "BV/RH", "aBevolz": "BV/RH", "psi": "B", "psipred": "B", "Bevolx": "B/R",
    "Bevoly": "B/R", "Bevolz": "B/R", "Bx": "B", "By": "B", "Bz": "B", "alphaloc": "1", "alpha1": "1",
    "u": "V", "v": "V", "w": "V", "au": "V2/H", "av": "V2/H", "aw": "V2/H", "ae": "V3/H", "x": "1", "y": "1",
    "z": "1",
    # diagnostic outputs: Cullen-Dehnen moments (x_ij m grad W ~ rho; dv, da
    # times m grad W), strain rates, limiter, density-pass sums
    "rho_sum": "R", "xilimiter": "1", "divvdt": "V2/H2", "arho": "RV/H", "grhox": "R/H", "grhoy": "R/H",
    "grhoz": "R/H", "dwdh": "R/H",
    **{f"cd_r{a}": "R" for a in ("xx", "xy", "xz", "yy", "yz", "zz")},
    **{f"cd_v{a}{b}": "RV/H" for a in "xyz" for b in "xyz"},
    **{f"cd_a{a}{b}": "RV2/H2" for a in "xyz" for b in "xyz"},
    **{f"dvdx_{a}{b}": "V/H" for a in "xyz" for b in "xyz"},
}


def scales(ic: dict, cs=None):
    V = max(float(np.max(np.abs(ic[k]))) for k in ("u", "v", "w"))
    if cs is not None:
        V = max(V, float(np.max(cs)))
    V = max(V, 1e-30)
    B = max(max(float(np.max(np.abs(ic[k]))) for k in ("Bx", "By", "Bz")), 1e-30)
    R = float(np.max(ic["rho"]))
    H = float(np.min(ic["h"]))
    return {"1": 1.0, "V": V, "V/H": V / H, "B/H": B / H, "RB/H": R * B / H, "VB/H": V * B / H,
            "BV/RH": B * V / (R * H), "B": B, "B/R": B / R, "V2/H": V * V / H, "V3/H": V ** 3 / H,
            "R": R, "R/H": R / H, "RV/H": R * V / H, "RV2/H2": R * V * V / (H * H), "V2/H2": V * V / (H * H)}


def max_rel(got, ref, name, sc):
    floor = sc[FAMILY[name]] if (sc is not None and name in FAMILY) else 0.0
    scale = max(float(np.max(np.abs(ref))), floor, 1e-300)
    return float(np.max(np.abs(got - ref))) / scale


# The Cullen-Dehnen switch is the roundoff-sensitive quantity: its limiter
# xi is 0/0 wherever div v and curl v both vanish, and alpha_loc / alpha1
# follow xi.  Only these fields may fall back to the reordering spread unless
# a test names more (the unjittered 2-D Orszag-Tang fixture, whose velocity
# field is stagnant along lines at t = 0, passes the switch's flips on to
# every evolved field after one step).
ROUNDOFF_SENSITIVE = frozenset(("alphaloc", "alpha1", "xilimiter"))


def _report(what, k, e, d_gpu, d_ref):
    path = os.environ.get("MHD_SPREAD_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"what": what, "field": k, "max_rel": e, "gpu": d_gpu, "spread": d_ref}) + "\n")


def assert_close(got: dict, ref: dict, names, rtol, sc=None, spread: dict | None = None, what="",
                 spread_fields=ROUNDOFF_SENSITIVE):
    """Every field within rtol of ref (relative to max(max|ref|, floor)).  A
    field of ``spread_fields`` that misses rtol passes when ||gpu - ref||_2
    <= 10 ||ref' - ref||_2, ref' being the reference summed in another order
    (``spread``); no other field has that fallback."""
    bad = []
    for k in names:
        e = max_rel(got[k], ref[k], k, sc)
        if e <= rtol:
            continue
        if spread is not None and k in spread and k in spread_fields:
            d_gpu = float(np.linalg.norm(got[k] - ref[k]))
            d_ref = float(np.linalg.norm(spread[k] - ref[k]))
            if d_ref > 0.0 and d_gpu <= 10.0 * d_ref:
                _report(what, k, e, d_gpu, d_ref)
                continue
            bad.append(f"{k}: max rel {e:.2e}; ||gpu-ref|| {d_gpu:.2e} vs reordering spread {d_ref:.2e}")
        else:
            bad.append(f"{k}: max rel {e:.2e} > {rtol:.0e}")
    assert not bad, f"{what}: " + "; ".join(bad)
