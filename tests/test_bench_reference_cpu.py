"""The reference arm of bench.py on the CPU: one JSON line in the contract's
shape, on the same metric, unit and workload as the B200 arm.

``bench.py --impl reference`` times the oracle (the reference's equations
restated in C, OpenMP) on the blast workload itself (--ref-n 0, the
default); it needs no GPU, so its line can be checked here on a small
lattice passed with --ref-n, which the line names in timed_workload.
"""

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_reference_arm_prints_one_contract_line():
    sys.path.insert(0, ROOT)
    import bench

    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "3", "--ref-n", "12"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT and d["higher_is_better"] is True
    assert d["config"]["workload"] == bench.blast_workload(128)
    # a sample smaller than the workload is named as such
    assert d["config"]["timed_workload"] == bench.blast_workload(12) and d["config"]["sample_particles"] == 12 ** 3
    assert d["steps"] == 2 and d["warmup"] == 3 and d["value"] > 0
    cpu = d["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
