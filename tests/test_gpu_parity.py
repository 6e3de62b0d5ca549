"""GPU parity: the CUDA path through the C ABI against the oracle (a CPU
restatement of the reference, pinned to the reference in test_oracle_pin.py).

Tolerances: FP64 solution and apply within 1e-12 relative of the oracle on
these sizes (their condition numbers keep both solvers' forward errors far
below that); an update must reproduce a from-scratch factorization of the new
matrix exactly (the kernels are deterministic and clean fronts are reused).
"""
import numpy as np
import pytest

import mf_oracle
from mfgpu import MF2D, MF3D, MFError, stencil
from problems import patch_update, problem, rel

pytestmark = pytest.mark.gpu

CASES = [
    (2, (31, 31), 4),
    (2, (127, 127), 4),       # the CPU-runnable workload's grid
    (2, (23, 57), 4),         # ragged
    (2, (130, 70), 4),        # remainder boxes
    (2, (63, 63), 8),
    (3, (15, 15, 15), 4),
    (3, (13, 17, 11), 3),     # ragged 3D
    (3, (31, 31, 31), 4),
]


def make(dim, N, A, ms, **kw):
    return MF2D(A, N[0], N[1], 1, ms, **kw) if dim == 2 else MF3D(A, N[0], N[1], N[2], 1, ms, **kw)


@pytest.mark.parametrize("dim,N,ms", CASES)
def test_factor_solve_apply_vs_oracle(dim, N, ms, lib):
    a, A, b = problem(dim, N, seed=11, nrhs=3)
    O = mf_oracle.MFOracle(A.to_scipy(), N, 1, ms)
    O.factor()
    F = make(dim, N, A, ms)
    F.Factor()
    X = F.Solve(b.T)
    Y = F.Apply(b.T)
    for r in range(b.shape[0]):
        xo = O.solve(b[r])
        yo = O.apply(b[r])
        assert rel(X[:, r], xo) < 1e-12
        assert rel(Y[:, r], yo) < 1e-13
        res = A.matvec(X[:, r]) - b[r]
        assert np.linalg.norm(res) / np.linalg.norm(b[r]) < 1e-12
    # single vector form equals the batched form bit for bit
    assert np.array_equal(F.Solve(b[0]), X[:, 0])


@pytest.mark.parametrize("dim,N,ms", [(2, (127, 127), 4), (2, (23, 57), 4), (3, (15, 15, 15), 4),
                                      (3, (31, 31, 31), 4)])
@pytest.mark.parametrize("same_kernels", [False, True])
def test_update_equals_refactor(dim, N, ms, same_kernels, monkeypatch):
    # An update may run a level's few dirty fronts on a different kernel than
    # the full factorization (cooperative instead of one CTA per front), which
    # changes the rounding but not the result.  With the kernel choice pinned
    # (MFGPU_FUSED_MIN_FRONTS=1: one CTA per front wherever it fits, in both
    # plans) the update reproduces a from-scratch factorization bit for bit.
    if same_kernels:
        monkeypatch.setenv("MFGPU_FUSED_MIN_FRONTS", "1")
    a, A, b = problem(dim, N, seed=21)
    side = 9 if dim == 2 else 4
    a2, _ = patch_update(a, N, side, 10.0, seed=3)
    A2 = stencil.build_laplacian(a2)
    mod = stencil.modified_dofs(A, A2)
    assert len(mod) > 0
    F = make(dim, N, A, ms)
    F.Factor()
    x_before = F.Solve(b[0])
    F.Update(A2, mod)
    st = F.stats()
    info = F.info()
    assert 0 < st["fronts"] < info["n_fronts"]     # only root paths were refactored
    x_upd = F.Solve(b[0])
    y_upd = F.Apply(b[0])
    G = make(dim, N, A2, ms)
    G.Factor()
    if same_kernels:
        assert np.array_equal(x_upd, G.Solve(b[0]))
        assert np.array_equal(y_upd, G.Apply(b[0]))
    else:
        assert rel(x_upd, G.Solve(b[0])) < 1e-13
        assert rel(y_upd, G.Apply(b[0])) < 1e-14
    # and against the oracle's own update
    O = mf_oracle.MFOracle(A.to_scipy(), N, 1, ms)
    O.factor()
    O.update(A2.to_scipy(), mod)
    assert rel(x_upd, O.solve(b[0])) < 1e-12
    assert rel(x_before, x_upd) > 1e-6


def test_apply_error_before_and_after_update_matches_reference_behaviour():
    # testProblemUpdating (test_src/DE/testMF2D.cpp:124-195): apply error of the
    # stale factor is large, after Update it is at rounding level.
    N = (127, 127)
    a = stencil.uniform_coefficients(N)
    a2 = a.copy()
    a2[:8, :8] *= 2
    A1 = stencil.build_laplacian(a)
    A2 = stencil.build_laplacian(a2)
    mod = stencil.modified_dofs(A1, A2)
    x = np.random.Generator(np.random.PCG64(1234)).random(A1.n)
    btrue = A2.matvec(x)
    F = MF2D(A1, 127, 127, 1, 8)
    F.Factor()
    e1 = rel(F.Apply(x), btrue)
    F.Update(A2, mod)
    e2 = rel(F.Apply(x), btrue)
    assert e1 > 1e-3
    assert e2 < 1e-14


def test_errors():
    a, A, b = problem(2, (31, 31), seed=2)
    with pytest.raises(RuntimeError):
        MF2D(A, 31, 31, 1, 40)        # recursion depth 1 (src/DE/mf2d.cpp:38-43)
    with pytest.raises(ValueError):
        MF2D(A, 30, 31, 1, 4)         # dimension mismatch
    F = MF2D(A, 31, 31, 1, 4)
    with pytest.raises(MFError):
        F.Solve(b[0])                 # before Factor
    # an indefinite matrix: negate the diagonal
    bad = stencil.CSR(A.row_ptr, A.col_ind, A.val.copy(), A.n)
    diag = np.repeat(np.arange(A.n), np.diff(A.row_ptr)) == A.col_ind
    bad.val[diag] *= -1
    G = MF2D(bad, 31, 31, 1, 4)
    with pytest.raises(MFError) as ei:
        G.Factor()
    assert ei.value.status == 6
    # the handle stays usable: a good factorization on the same process works
    F.Factor()
    assert rel(A.matvec(F.Solve(b[0])), b[0]) < 1e-13


@pytest.fixture
def env_var(monkeypatch):
    """Set an MFGPU_* switch for the handles created inside the test."""
    def set_(name, value):
        monkeypatch.setenv(name, str(value))
    return set_


@pytest.mark.parametrize("dim,N,ms", [(2, (127, 127), 4), (2, (130, 70), 4), (3, (15, 15, 15), 4),
                                      (3, (13, 17, 11), 3), (3, (31, 31, 31), 4)])
@pytest.mark.parametrize("nrhs", [1, 3, 9])
def test_cooperative_sweeps_vs_oracle(dim, N, ms, nrhs, env_var):
    # every level of at most 256 fronts through the multi-CTA blocked sweeps
    env_var("MFGPU_SOLVE_COOP_MIN_N", 1)
    a, A, b = problem(dim, N, seed=13, nrhs=nrhs)
    F = make(dim, N, A, ms)
    F.Factor()
    X = F.Solve(b.T)
    O = mf_oracle.MFOracle(A.to_scipy(), N, 1, ms)
    O.factor()
    for r in range(nrhs):
        assert rel(X[:, r], O.solve(b[r])) < 1e-12
    env_var("MFGPU_SOLVE_COOP_MIN_N", 0)
    G = make(dim, N, A, ms)
    G.Factor()
    Xg = G.Solve(b.T)
    assert rel(X, Xg) < 1e-13
    assert np.array_equal(F.Solve(b.T), X)      # deterministic


@pytest.mark.parametrize("dim,N,ms", [(2, (255, 255), 4), (2, (130, 70), 4), (3, (31, 31, 31), 4),
                                      (3, (13, 17, 11), 3)])
@pytest.mark.parametrize("kernel", ["panel", "coop"])
def test_level_kernels_vs_oracle(dim, N, ms, kernel, env_var):
    """Levels of moderate fronts factored panel by panel (k_diag_factor +
    k_panel_trsm + k_trail_syrk, MFGPU_PANEL_MAX_N=4096) or by the cooperative
    kernel (the default): both within 1e-12 of the oracle, before and after a
    localized update."""
    env_var("MFGPU_PANEL_MAX_N", 4096 if kernel == "panel" else 0)
    a, A, b = problem(dim, N, seed=17, nrhs=2)
    F = make(dim, N, A, ms)
    F.profile(True)
    F.Factor()
    X = F.Solve(b.T)
    O = mf_oracle.MFOracle(A.to_scipy(), N, 1, ms)
    O.factor()
    for r in range(2):
        assert rel(X[:, r], O.solve(b[r])) < 1e-12
    side = 9 if dim == 2 else 4
    a2, _ = patch_update(a, N, side, 10.0, seed=5)
    A2 = stencil.build_laplacian(a2)
    mod = stencil.modified_dofs(A, A2)
    F.Update(A2, mod)
    O.update(A2.to_scipy(), mod)
    X2 = F.Solve(b.T)
    for r in range(2):
        assert rel(X2[:, r], O.solve(b[r])) < 1e-12
