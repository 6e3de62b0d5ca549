"""The C++ drop-in: callers of the reference's API (linalg.hpp + mf.hpp) switch
to the B200 path without source changes.

CPU: tests/cpp/test_dropin.cpp compiles and links against the drop-in headers
and libmfgpu.so; where the reference sources are present, its own drivers
test_src/DE/testMF2D.cpp and testMF3D.cpp compile unchanged against them.
GPU: both run and report rounding-level errors.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "updating-multifrontal_b200")


def _reference_dir():
    """Where the reference sources are: the REF variable of oracle/Makefile
    (the environment's REF overrides its default, as make does)."""
    p = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"],
                       capture_output=True, text=True)
    return p.stdout.strip() if p.returncode == 0 else ""


REF = _reference_dir()
REFBIN = os.path.join(ROOT, "oracle", "_ref")
FLAGS = ["-O2", "-std=c++17", f"-I{PKG}/include/LinAlg", f"-I{PKG}/include/DE",
         f"-I{ROOT}/include", f"-I{ROOT}/tests/cpp"]
LINK = [f"-L{PKG}/lib", "-lmfgpu", f"-Wl,-rpath,{PKG}/lib"]


def compile_dropin(out):
    subprocess.run(["g++"] + FLAGS + [os.path.join(ROOT, "tests/cpp/test_dropin.cpp")] + LINK +
                   ["-o", out], check=True, capture_output=True, text=True)


def test_dropin_driver_compiles_and_links(tmp_path, lib):
    compile_dropin(str(tmp_path / "t"))


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "test_src")),
                    reason="reference sources not present")
@pytest.mark.parametrize("drv", ["testMF2D.cpp", "testMF3D.cpp"])
def test_reference_drivers_compile_unchanged(tmp_path, drv, lib):
    subprocess.run(["g++", "-O2", "-std=c++11", "-w", f"-I{PKG}/include/LinAlg",
                    f"-I{PKG}/include/DE", f"-I{ROOT}/include", f"-I{REF}/test_include/DE",
                    os.path.join(REF, "test_src/DE", drv)] + LINK + ["-o", str(tmp_path / "d")],
                   check=True, capture_output=True, text=True)


@pytest.mark.gpu
def test_dropin_driver_runs(tmp_path, lib):
    exe = str(tmp_path / "t")
    compile_dropin(exe)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(p.stdout)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "PASSED" in p.stdout


def _numbers_after(text, label):
    m = re.findall(re.escape(label) + r"\s*\n\s*([0-9.eE+-]+)", text)
    return [float(x) for x in m]


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.isfile(os.path.join(REFBIN, "dropin_testMF2D")),
                    reason="reference drivers were not built against the drop-in headers")
def test_reference_test_drivers_run_on_the_gpu_path():
    # testProblemUniform + testProblemUpdating (test_src/DE/testMF2D.cpp:39-85)
    p = subprocess.run([os.path.join(REFBIN, "dropin_testMF2D"), "127", "127", "1"],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    out = p.stdout
    assert _numbers_after(out, "Relative apply error is:")[0] < 1e-14
    assert _numbers_after(out, "Relative solve error is:")[0] < 1e-12
    assert _numbers_after(out, "Relative apply error without updating is:")[0] > 1e-3
    assert _numbers_after(out, "Relative apply error after updating is:")[0] < 1e-14
    p = subprocess.run([os.path.join(REFBIN, "dropin_testMF3D"), "23", "23", "23", "1"],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    out = p.stdout
    assert _numbers_after(out, "Relative apply error after updating is:")[-1] < 1e-14
