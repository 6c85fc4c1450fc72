"""Loading helpers for the golden fixtures in ``tests/golden``."""

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("ot2d", "shock2d", "blast3d", "ref_orstang3d")


def load(case):
    d = np.load(os.path.join(GOLDEN, f"{case}.npz"))
    params = json.loads(str(d["params"]))
    return d, params


def section(d, prefix):
    return {k[len(prefix) + 1:]: d[k] for k in d.files if k.startswith(prefix + "/")}
