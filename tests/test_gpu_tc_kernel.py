"""GPU: the tensor-core update kernels against an FP64 CPU reference
(tests/cpp/tc_kernel_check.cu, compiled with nvcc for sm_100a and run)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def test_tc_update_matches_fp64_reference(tmp_path):
    # nvcc ships with the image; a missing compiler is a failure, not a skip
    assert shutil.which("nvcc"), "nvcc not found on PATH"
    exe = str(tmp_path / "tc_kernel_check")
    subprocess.run(["nvcc", "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                    os.path.join(ROOT, "tests", "cpp", "tc_kernel_check.cu"), "-o", exe],
                   check=True, capture_output=True, text=True, timeout=900)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-4000:] + out.stderr[-2000:]
    assert out.stdout.rstrip().endswith("ok")
