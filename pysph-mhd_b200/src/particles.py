"""Particle property names of the SPMHD scheme.

The names are the reference's (``src/particles.py``): a user's case code and
output readers keep working.  Grouping follows the reference -- base
properties (``:1-51``), output properties (``:53-71``), evolved magnetic
state (``:73-78``), internals (``:80-99``), Cullen-Dehnen moments
(``:101-129``) and strain diagnostics (``:131-141``).
"""

BASE_PROPERTIES = tuple(
    "x y z gid tag".split()
) + ({"name": "itype", "type": "int", "default": 1},) + tuple(
    "u v w rho rho_sum h m cs p e au av aw arho ae ah x0 y0 z0 u0 v0 w0 upred vpred wpred epred e0 h0 div "
    "dt_cfl dt_force dt_adapt grhox grhoy grhoz dwdh omega converged alpha1 alpha10 Bx By Bz".split()
)

OUTPUT_PROPERTIES = tuple("x y z gid u v w rho h m itype alpha1 p e Bx By Bz".split())

_STATE_PROPERTIES = tuple("Bevolx Bevoly Bevolz psi".split())

_INTERNAL_PROPERTIES = tuple(
    "Bevolxpred Bevolypred Bevolzpred psipred Bxpred Bypred Bzpred aBevolx aBevoly aBevolz apsi "
    "Bevolx0 Bevoly0 Bevolz0 psi0 divBsymm divBdiff div_for_psi".split()
)

_CULLEN_DEHNEN_PROPERTIES = ("alphaloc", "xilimiter", "divvdt") + tuple(
    f"cd_{k}" for k in "rxx rxy rxz ryy ryz rzz".split()
) + tuple(f"cd_{q}{a}{b}" for q in "va" for a in "xyz" for b in "xyz")

_CURRENT_STRAIN_PROPERTIES = tuple(f"dvdx_{a}{b}" for a in "xyz" for b in "xyz")

PROPERTIES = _STATE_PROPERTIES + _INTERNAL_PROPERTIES + _CULLEN_DEHNEN_PROPERTIES + _CURRENT_STRAIN_PROPERTIES

# (predicted, current) pairs synchronised before the warm-up RHS
INITIAL_PREDICTOR_PAIRS = (
    ("Bevolxpred", "Bevolx"),
    ("Bevolypred", "Bevoly"),
    ("Bevolzpred", "Bevolz"),
    ("psipred", "psi"),
    ("upred", "u"),
    ("vpred", "v"),
    ("wpred", "w"),
    ("epred", "e"),
)

INITIAL_STATE_GPU_PROPERTIES = ("Bx", "By", "Bz", *_STATE_PROPERTIES, *(p for p, _ in INITIAL_PREDICTOR_PAIRS))


def property_names():
    """Every property name, int ``itype`` included."""
    out = []
    for p in BASE_PROPERTIES + PROPERTIES:
        out.append(p["name"] if isinstance(p, dict) else p)
    return out
