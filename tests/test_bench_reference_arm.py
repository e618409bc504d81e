"""bench.py's reference arm on CPU: planned, counted and timed by the oracle alone.

The arm times the CPU restatement of the reference executor and must never load the product library, so the
ratio between the two arms compares independent implementations.  Run here on a small instance of the same
workload family (rand3reg n = 64, target 2^8) so that it ends in seconds.
"""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_runs_without_the_product_library():
    proc = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--nodes", "64", "--target-log2", "8",
                           "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert proc.returncode == 0, proc.stderr[-2000:]
    line = json.loads([l for l in proc.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["product_library_loaded"] is False
    assert line["config"]["planned_by"] == "oracle greedy + find_slices_to_size"
    assert line["config"]["n_slices"] >= 16
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
