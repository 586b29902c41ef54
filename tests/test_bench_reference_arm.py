"""bench.py --impl reference runs the reference's own step on the workload's
configuration without ever loading the CUDA library: its input comes from
the oracle's restatement of the driver's Voronoi construction, and the
process's memory map is checked after the arm has run (a small cube here;
the arm's logic does not depend on the size)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--size", "24", "--grains", "12", "--steps", "2",
            "--warmup", "1", "--no-cpu"]
sys.path.insert(0, ".")
import bench
bench.main()
maps = open("/proc/self/maps").read()
print("MAPS", json.dumps({"gpk_b200": "libgpk_b200.so" in maps, "ref": "libgpk_ref.so" in maps}))
"""


def test_reference_arm_never_loads_the_library(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference harness not built")
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    maps = json.loads([l for l in r.stdout.splitlines() if l.startswith("MAPS ")][0][5:])
    line = json.loads(lines[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["steps"] == 2 and line["warmup"] == 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["config"]["cells"] == 24 ** 3
    assert maps == {"gpk_b200": False, "ref": True}
