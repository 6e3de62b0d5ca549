"""mfgpu_solve_device_noalloc: the solve for callers that may not allocate
device memory at solve time (a service holding a fixed device-memory budget
from start-up, or a loop that cannot afford cudaMalloc's implicit device-wide
synchronisation).  It must give the same answer as the allocating
mfgpu_solve_device, call after call, while using only the library's fixed
32 MiB scratch array.

This file is named to be collected last, so a stop-at-first-failure run has
already run every other test; it also passes alone in a fresh process (its
first call does the per-device set-up).
"""
import ctypes as C

import numpy as np
import pytest

from mfgpu import MF2D, _lib
from problems import problem

pytestmark = pytest.mark.gpu


def _fn():
    lib = _lib.load()
    f = lib.mfgpu_solve_device_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int64]
    f.restype = C.c_int
    return lib, f


def test_noalloc_solve_matches_allocating_solve_twice():
    import torch

    lib, noalloc = _fn()
    N = (127, 127)
    _, A, b = problem(2, N, seed=31, nrhs=3)
    n, nrhs = A.n, b.shape[0]
    F = MF2D(A, N[0], N[1], 1, 4)
    F.Factor()
    db = torch.from_numpy(np.ascontiguousarray(b)).cuda()     # n x nrhs column-major, ld = n
    ref = torch.empty_like(db)
    F.solve_device(db.data_ptr(), ref.data_ptr(), nrhs, n)
    torch.cuda.synchronize()
    ref_h = ref.cpu().numpy()
    for call in range(2):
        out = torch.full_like(db, float("nan"))
        st = noalloc(F._h, db.data_ptr(), out.data_ptr(), nrhs, n)
        assert st == 0, lib.mfgpu_last_error(F._h).decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        for r in range(nrhs):
            err = np.linalg.norm(got[r] - ref_h[r]) / np.linalg.norm(ref_h[r])
            assert err < 1e-12, (call, r, err)
        # and it is a solution: FP64 residual of the 5-point system
        res = np.linalg.norm(A.matvec(got[0]) - b[0]) / np.linalg.norm(b[0])
        assert res < 1e-12


def test_noalloc_rejects_problems_beyond_the_scratch():
    lib, noalloc = _fn()
    # 2D 1200 x 1200 with leaf parameter 8 needs about 38.8 MiB of workspace
    # per right-hand side, more than the 32 MiB array; the size check comes
    # before anything touches the device.
    from mfgpu import stencil
    N = (1200, 1200)
    A = stencil.build_laplacian(stencil.uniform_coefficients(N))
    F = MF2D(A, N[0], N[1], 1, 8)
    st = noalloc(F._h, C.c_void_p(16), C.c_void_p(16), 1, A.n)
    assert st == _lib.MFGPU_ERR_ARG
    msg = lib.mfgpu_last_error(F._h).decode()
    assert "too large" in msg and "MiB" in msg
