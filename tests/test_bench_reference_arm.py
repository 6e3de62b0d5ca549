"""CPU: bench.py's reference arm runs the reference's own code only.  It prints
one JSON line with the metric, its sample and the work counted from the
reference's front sizes, and the process never maps a shared object of the
product (libmfgpu.so)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import sys, runpy
sys.argv = ["bench.py", "--impl", "reference", "--workload", "2d-127", "--steps", "1",
            "--warmup", "1"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    assert not e.code, e.code
maps = open("/proc/self/maps").read()
print("MAPPED_PRODUCT" if "libmfgpu" in maps else "CLEAN")
"""


def test_reference_arm_maps_no_product_library():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refio
    if not refio.have_reference():
        pytest.fail("reference harness oracle/_ref/ref_harness is not built")
    p = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    lines = p.stdout.strip().splitlines()
    assert lines[-1] == "CLEAN"
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["unit"] == "TFLOP/s" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["flops_per_step"]["factor"] > 0 and line["flops_per_step"]["update"] > 0
