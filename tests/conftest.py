import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "updating-multifrontal_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def lib():
    """libmfgpu.so, built in-tree (nvcc cross-compiles without a GPU) if missing."""
    import subprocess
    from mfgpu import _lib
    if not os.path.isfile(_lib.LIB_PATH):
        subprocess.run(["make", "-j", "8"], cwd=PKG, check=True, capture_output=True)
    return _lib.load()
