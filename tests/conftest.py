"""Test configuration: the ``gpu`` marker and import paths.

``-m "not gpu"`` runs the oracle-vs-golden checks, host logic and C-ABI
symbol checks on CPU; ``-m gpu`` runs the CUDA parity tests.
"""

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pysph-mhd_b200")
BUILD_DIR = PKG
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
