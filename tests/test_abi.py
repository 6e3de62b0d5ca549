"""The C ABI library: it loads, exports every function include/mfgpu.h
declares, and its host-only parts work without a GPU.  Compute entry points
never fall back to the CPU: without a usable device they fail."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from mfgpu import Symbolic, _lib, stencil

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "mfgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mfgpu_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 25
    for nm in names:
        assert hasattr(lib, nm), nm
    assert set(names) <= set(_lib.EXPORTED)


def test_status_strings_and_options(lib):
    assert _lib.status_string(0) == "ok"
    assert "SPD" in _lib.status_string(6)
    o = _lib.default_options()
    assert o.precision == _lib.MFGPU_FP64 and o.refine_tol == 1e-10


def test_symbolic_errors_match_reference():
    with pytest.raises(RuntimeError):
        Symbolic(2, (31, 31), 1, 40)        # recursion depth 1, src/DE/mf2d.cpp:38-43
    with pytest.raises(ValueError):
        Symbolic(4, (31, 31), 1, 4)


def test_symbolic_sizes_2d_1023():
    S = Symbolic(2, (1023, 1023), 1, 8)
    assert S.levels == 7 and S.ndof == 1023 * 1023
    assert S.n_fronts == sum(4 ** l for l in range(7))
    root = S.front(0)
    assert root["n"] == 2045 and root["m"] == 0


def test_compute_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    A = stencil.build_laplacian(stencil.uniform_coefficients((31, 31)))
    from mfgpu import MF2D, MFError
    with pytest.raises(MFError) as ei:
        MF2D(A, 31, 31, 1, 4)
    assert ei.value.status == _lib.MFGPU_ERR_CUDA


def test_nonsymmetric_matrix_rejected_before_any_device_work():
    # the factorization reads the lower triangle only: a nonsymmetric matrix
    # is refused at creation (on any machine, GPU or not)
    A = stencil.build_laplacian(stencil.uniform_coefficients((31, 31)))
    from mfgpu import MF2D
    bad = stencil.CSR(A.row_ptr, A.col_ind, A.val.copy(), A.n)
    off = np.flatnonzero(np.repeat(np.arange(A.n), np.diff(A.row_ptr)) != A.col_ind)[7]
    bad.val[off] *= 1.01
    with pytest.raises(ValueError, match="not symmetric"):
        MF2D(bad, 31, 31, 1, 4)
