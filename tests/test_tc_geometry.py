"""Host-only check of the tensor-core update's tile bookkeeping
(csrc/kernels_tc.cu): tiles per front, tile-index decoding and pack capacity
against a brute-force enumeration, compiled with nvcc and run on the CPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tile_enumeration_matches_brute_force(tmp_path):
    # nvcc ships with the image; a missing compiler is a failure, not a skip
    assert shutil.which("nvcc"), "nvcc not found on PATH"
    exe = str(tmp_path / "tc_geometry")
    subprocess.run(["nvcc", "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
                    os.path.join(ROOT, "tests", "cpp", "tc_geometry.cu"), "-o", exe],
                   check=True, capture_output=True, text=True, timeout=600)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok")
