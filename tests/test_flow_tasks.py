"""Host-only check of the flag-ordered sweeps' task lists
(csrc/kernels_solve.cu flow_tasks): every task listed once, flag offsets per
front, and every wait on a flag raised by a task listed earlier (the property
that keeps the persistent cooperative grid from stalling); compiled with nvcc
and run on the CPU."""
import os
import shutil
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_flow_task_order_has_no_forward_waits(tmp_path):
    # nvcc ships with the image; a missing compiler is a failure, not a skip
    assert shutil.which("nvcc"), "nvcc not found on PATH"
    exe = str(tmp_path / "flow_tasks_check")
    subprocess.run(["nvcc", "-std=c++17", "-O1", "--expt-relaxed-constexpr", "-gencode",
                    "arch=compute_100a,code=sm_100a",
                    os.path.join(ROOT, "tests", "cpp", "flow_tasks_check.cu"), "-o", exe],
                   check=True, capture_output=True, text=True, timeout=900)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok")
