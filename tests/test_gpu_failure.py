"""Failure paths that fault, trap and hang nothing (the reference has none: its
LAPACK failures abort through assert, include/LinAlg/dense.hpp:187).

* Bounded device waits: with a poll limit of one, the cooperative kernels'
  grid barriers give up at once (CTAs with no first-block work arrive long
  before the others), the kernel records the timeout in its error word and
  returns, and the call reports MFGPU_ERR_TIMEOUT.  With the built-in limit
  restored the same handle factors and solves exactly as a fresh one.
* Injected device allocation failures (host side): every allocation point of
  handle creation and of the first solve fails cleanly with MFGPU_ERR_OOM,
  leaks nothing, and the next call succeeds.
"""
import numpy as np
import pytest

from mfgpu import MF2D, MFError, _lib, inject_alloc_failure
from problems import problem

pytestmark = pytest.mark.gpu

N = (255, 255)


@pytest.fixture(scope="module")
def prob():
    _, A, b = problem(2, N, seed=41, nrhs=2)
    ref = MF2D(A, N[0], N[1], 1, 4)
    ref.Factor()
    x = ref.Solve(b.T)
    ref.close()
    return A, b, x


def test_barrier_timeout_in_factor_then_recovers(prob, monkeypatch):
    A, b, x = prob
    monkeypatch.setenv("MFGPU_PANEL_MAX_N", "0")   # levels on the cooperative (grid-barrier) kernel
    F = MF2D(A, N[0], N[1], 1, 4)
    F.set_wait_limit(1)
    with pytest.raises(MFError) as e:
        F.Factor()
    assert e.value.status == _lib.MFGPU_ERR_TIMEOUT
    assert "grid barrier" in str(e.value)
    with pytest.raises(MFError) as e:        # not factored: Solve is refused
        F.Solve(b[0])
    assert e.value.status == _lib.MFGPU_ERR_STATE
    F.set_wait_limit(0)
    F.Factor()
    np.testing.assert_array_equal(F.Solve(b.T), x)   # bit for bit: same kernels, same order


def test_barrier_timeout_in_cooperative_sweeps_then_recovers(prob, monkeypatch):
    A, b, _ = prob
    monkeypatch.setenv("MFGPU_SOLVE_COOP_MIN_N", "256")   # top levels use the cooperative sweeps
    F = MF2D(A, N[0], N[1], 1, 4)
    F.Factor()
    x0 = F.Solve(b.T)
    F.set_wait_limit(1)
    with pytest.raises(MFError) as e:
        F.Solve(b.T)
    assert e.value.status == _lib.MFGPU_ERR_TIMEOUT
    F.set_wait_limit(0)
    np.testing.assert_array_equal(F.Solve(b.T), x0)
    res = np.linalg.norm(A.matvec(x0[:, 0]) - b[0]) / np.linalg.norm(b[0])
    assert res < 1e-12


def test_injected_allocation_failures_in_create_and_solve(prob):
    import torch

    A, b, x = prob
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    failures = 0
    try:
        for k in range(200):
            inject_alloc_failure(k)
            try:
                F = MF2D(A, N[0], N[1], 1, 4)
            except MFError as e:
                assert e.status == _lib.MFGPU_ERR_OOM and "injected" in str(e)
                failures += 1
                continue
            break
        else:
            pytest.fail("handle creation never succeeded")
    finally:
        inject_alloc_failure(-1)
    assert failures == k and failures >= 10      # every allocation point of creation was hit
    F.close()
    torch.cuda.synchronize()
    leaked = free0 - torch.cuda.mem_get_info()[0]
    assert leaked <= 2 << 20, f"{leaked} bytes not returned after failed creations"

    F = MF2D(A, N[0], N[1], 1, 4)
    F.Factor()
    inject_alloc_failure(0)                       # the first solve allocates its workspace
    try:
        with pytest.raises(MFError) as e:
            F.Solve(b.T)
        assert e.value.status == _lib.MFGPU_ERR_OOM
    finally:
        inject_alloc_failure(-1)
    np.testing.assert_array_equal(F.Solve(b.T), x)
