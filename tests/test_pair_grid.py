"""The derivative forms' neighbour search, on the CPU.

The forward-mode and adjoint passes find neighbours by walking a uniform
cell grid (``csrc/mhd_pairgrid.cuh``).  ``tests/pair_grid_check.cu`` runs the
same plan, key and walk functions on the host for random particle sets --
2-D and 3-D, periodic and open axes, wide and narrow boxes, spread and
outsized smoothing lengths, several slice counts -- and checks that each
particle's reported pairs are exactly the brute-force ones, each once.
"""

import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not available")
def test_grid_walk_finds_exactly_the_brute_force_pairs(tmp_path):
    exe = str(tmp_path / "pair_grid_check")
    cmd = [NVCC, "-std=c++17", "-O2", "-Xcompiler", "-ffp-contract=off", "-Wno-deprecated-gpu-targets",
           "-diag-suppress", "20013", "-I",
           os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "pysph-mhd_b200", "csrc"),
           os.path.join(HERE, "pair_grid_check.cu"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, timeout=600)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    fields = out.stdout.split()
    assert fields[0] == "ok", out.stdout
    # the check is not vacuous: many pairs, and grids of many cells
    assert int(fields[fields.index("pairs") + 1]) > 100000, out.stdout
    assert int(fields[fields.index("cells_max") + 1]) > 100, out.stdout
