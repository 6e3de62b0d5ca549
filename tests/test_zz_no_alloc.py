"""mfgpu_solve_device_noalloc: the solve for callers that may not allocate
device memory at solve time (a service holding a fixed device-memory budget
from start-up, or a loop that cannot afford cudaMalloc's implicit device-wide
synchronisation).  It must give the same answer as the allocating
mfgpu_solve_device, call after call, while using only the library's fixed
32 MiB scratch array: on a freshly factored handle, whose solve workspace has
never been allocated, the device's free memory must not change across a call.

This file is named to be collected last, so a stop-at-first-failure run has
already run every other test; it also passes alone in a fresh process (the
first call on a device does the per-device set-up).
"""
import ctypes as C

import numpy as np
import pytest

from mfgpu import MF2D, _lib
from problems import problem

pytestmark = pytest.mark.gpu


def _fn():
    lib = _lib.load()
    return lib, lib.mfgpu_solve_device_noalloc


def _columns(torch, b, ld):
    """b (nrhs, n) as a device buffer of nrhs columns with leading dimension ld."""
    nrhs, n = b.shape
    buf = torch.full((nrhs, ld), float("nan"), dtype=torch.float64, device="cuda")
    buf[:, :n] = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    return buf


def _check(got, ref, tol=1e-12):
    for r in range(ref.shape[0]):
        err = np.linalg.norm(got[r] - ref[r]) / np.linalg.norm(ref[r])
        assert err < tol, (r, err)


def test_noalloc_solve_matches_allocating_solve_twice():
    import torch

    lib, noalloc = _fn()
    N = (127, 127)
    _, A, b = problem(2, N, seed=31, nrhs=3)
    n, nrhs = A.n, b.shape[0]
    # the allocating solve on its own handle
    G = MF2D(A, N[0], N[1], 1, 4)
    G.Factor()
    db = torch.from_numpy(np.ascontiguousarray(b)).cuda()     # n x nrhs column-major, ld = n
    ref = torch.empty_like(db)
    G.solve_device(db.data_ptr(), ref.data_ptr(), nrhs, n)
    torch.cuda.synchronize()
    ref_h = ref.cpu().numpy()
    # the no-allocation solve first on a fresh handle, then again
    F = MF2D(A, N[0], N[1], 1, 4)
    F.Factor()
    for call in range(2):
        out = torch.full_like(db, float("nan"))
        st = noalloc(F._h, db.data_ptr(), out.data_ptr(), nrhs, n)
        assert st == 0, lib.mfgpu_last_error(F._h).decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        _check(got, ref_h)
        # and it is a solution: FP64 residual of the 5-point system
        res = np.linalg.norm(A.matvec(got[0]) - b[0]) / np.linalg.norm(b[0])
        assert res < 1e-12


def test_noalloc_allocates_nothing_chunks_strides_and_cooperative_sweeps(monkeypatch):
    """20 right-hand sides (two chunks of at most 16) in buffers with leading
    dimension above n, in place and out of place, on a grid whose top levels
    use the cooperative sweeps (their size rule lowered to 256 unknowns)."""
    import torch

    lib, noalloc = _fn()
    monkeypatch.setenv("MFGPU_SOLVE_COOP_MIN_N", "256")
    N = (255, 255)
    _, A, b = problem(2, N, seed=37, nrhs=20)
    n, nrhs, ld = A.n, b.shape[0], A.n + 37
    G = MF2D(A, N[0], N[1], 1, 4)
    G.Factor()
    ref = G.Solve(b.T).T                                      # (nrhs, n), allocating path

    # per-device set-up of the scratch address happens on the first call in the
    # process; make it on a throw-away handle so the measured call below is a
    # plain one
    H = MF2D(A, N[0], N[1], 1, 4)
    H.Factor()
    warm = _columns(torch, b[:1], ld)
    assert noalloc(H._h, warm.data_ptr(), warm.data_ptr(), 1, ld) == 0
    H.close()

    F = MF2D(A, N[0], N[1], 1, 4)                             # fresh: no solve workspace yet
    F.Factor()
    src = _columns(torch, b, ld)
    dst = torch.full_like(src, float("nan"))
    inplace = _columns(torch, b, ld)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st = noalloc(F._h, src.data_ptr(), dst.data_ptr(), nrhs, ld)
    free1 = torch.cuda.mem_get_info()[0]
    assert st == 0, lib.mfgpu_last_error(F._h).decode()
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    st = noalloc(F._h, inplace.data_ptr(), inplace.data_ptr(), nrhs, ld)
    assert st == 0, lib.mfgpu_last_error(F._h).decode()
    torch.cuda.synchronize()
    _check(dst[:, :n].cpu().numpy(), ref)
    _check(inplace[:, :n].cpu().numpy(), ref)
    # the padding rows past n are left alone
    assert torch.isnan(dst[:, n:]).all().item()
    # the call reports its own timing and work
    stats = F.stats()
    assert stats["seconds"] > 0 and stats["flops"] > 0


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
