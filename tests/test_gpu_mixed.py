"""GPU: the mixed-precision path (FP32 factorization with symmetric diagonal
scaling, FP64 residuals and preconditioned conjugate-gradient refinement).

Tolerances: every solve must reach ||b - A x|| / ||b|| <= 1e-10 (the
refinement target); its solution then agrees with the FP64 path to within
cond(A) * 1e-10, bounded here by 1e-6 for these coefficient contrasts.  The
mixed Apply applies the FP32 factorization, so it matches the FP64 Apply to
single-precision accuracy (5e-5 relative).
"""
import numpy as np
import pytest

from mfgpu import MF2D, MF3D, MFGPU_MIXED, MFError, stencil
from problems import patch_update, problem, rel

pytestmark = pytest.mark.gpu

TOL = 1e-10

CASES = [
    (2, (31, 31), 4),
    (2, (127, 127), 4),
    (2, (23, 57), 4),
    (2, (255, 255), 8),
    (3, (15, 15, 15), 4),
    (3, (13, 17, 11), 3),
    (3, (31, 31, 31), 4),
]


def make(dim, N, A, ms, **kw):
    return MF2D(A, N[0], N[1], 1, ms, **kw) if dim == 2 else MF3D(A, N[0], N[1], N[2], 1, ms, **kw)


def relres(A, x, b):
    return float(np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b))


@pytest.fixture(params=["default", "tensor-core levels", "tensor-core sub-panels", "panel levels"])
def tc_mode(request, monkeypatch):
    """'tensor-core levels' sends every level with a front of 512 or more onto
    the tcgen05 trailing update (three-term TF32) with their 128-column
    sub-panels factored by the cooperative kernel; 'tensor-core sub-panels'
    the same with the sub-panels by k_diag_factor + k_panel_trsm (the
    default); 'panel levels' factors every level of fronts up to 4096 panel
    by panel (k_diag_factor + k_panel_trsm + k_trail_syrk)."""
    if request.param.startswith("tensor-core"):
        monkeypatch.setenv("MFGPU_TC_MIN_N", "512")
    if request.param == "tensor-core levels":
        monkeypatch.setenv("MFGPU_SUBPANEL", "0")
    if request.param == "panel levels":
        monkeypatch.setenv("MFGPU_PANEL_MAX_N", "4096")
    return request.param


@pytest.mark.parametrize("dim,N,ms", CASES)
def test_mixed_solve_reaches_tolerance(dim, N, ms, tc_mode):
    a, A, b = problem(dim, N, seed=31, nrhs=3)
    M = make(dim, N, A, ms, precision=MFGPU_MIXED, refine_tol=TOL)
    M.Factor()
    X = M.Solve(b.T)
    st = M.stats()
    assert st["residual"] <= TOL
    assert 1 <= st["iterations"] <= 50
    D = make(dim, N, A, ms)
    D.Factor()
    Xd = D.Solve(b.T)
    for r in range(b.shape[0]):
        assert relres(A, X[:, r], b[r]) <= 2 * TOL     # host FP64 residual agrees
        assert rel(X[:, r], Xd[:, r]) < 1e-6
    # deterministic: a second solve is bit-identical
    assert np.array_equal(M.Solve(b.T), X)
    # Apply of the FP32 factorization
    Y = M.Apply(b.T)
    Yd = D.Apply(b.T)
    for r in range(b.shape[0]):
        assert rel(Y[:, r], Yd[:, r]) < 5e-5
    info = M.info()
    assert info["front_bytes"] * 2 == D.info()["front_bytes"]    # FP32 arenas


@pytest.mark.parametrize("dim,N,ms", [(2, (127, 127), 4), (3, (31, 31, 31), 4)])
def test_mixed_update(dim, N, ms, tc_mode):
    a, A, b = problem(dim, N, seed=41)
    side = 9 if dim == 2 else 4
    a2, _ = patch_update(a, N, side, 10.0, seed=5)
    A2 = stencil.build_laplacian(a2)
    mod = stencil.modified_dofs(A, A2)
    M = make(dim, N, A, ms, precision=MFGPU_MIXED)
    M.Factor()
    x1 = M.Solve(b[0])
    assert relres(A, x1, b[0]) <= 2 * TOL
    M.Update(A2, mod)
    assert 0 < M.stats()["fronts"] < M.info()["n_fronts"]
    x2 = M.Solve(b[0])
    assert M.stats()["residual"] <= TOL
    assert relres(A2, x2, b[0]) <= 2 * TOL
    assert rel(x1, x2) > 1e-6
    # the updated factorization is as good a preconditioner as a fresh one
    G = make(dim, N, A2, ms, precision=MFGPU_MIXED)
    G.Factor()
    G.Solve(b[0])
    assert M.stats()["iterations"] <= G.stats()["iterations"] + 2


def test_mixed_not_converged_reports():
    a, A, b = problem(2, (63, 63), seed=7)
    M = MF2D(A, 63, 63, 1, 4, precision=MFGPU_MIXED, refine_tol=1e-30, refine_maxit=2)
    M.Factor()
    with pytest.raises(MFError) as ei:
        M.Solve(b[0])
    assert ei.value.status == 9
    # the handle stays usable with a reachable target
    N = MF2D(A, 63, 63, 1, 4, precision=MFGPU_MIXED)
    N.Factor()
    assert relres(A, N.Solve(b[0]), b[0]) <= 2 * TOL


def test_mixed_indefinite_fails_loudly():
    a, A, b = problem(2, (31, 31), seed=2)
    bad = stencil.CSR(A.row_ptr, A.col_ind, A.val.copy(), A.n)
    diag = np.repeat(np.arange(A.n), np.diff(A.row_ptr)) == A.col_ind
    bad.val[diag] *= -1
    G = MF2D(bad, 31, 31, 1, 4, precision=MFGPU_MIXED)
    with pytest.raises(MFError) as ei:
        G.Factor()
    assert ei.value.status == 6


@pytest.mark.parametrize("split", [1, 3])
def test_tensor_core_split_forms(split, monkeypatch):
    # plain TF32 (split 1) needs more refinement iterations than the three-term
    # form but reaches the same tolerance
    monkeypatch.setenv("MFGPU_TC_MIN_N", "512")
    monkeypatch.setenv("MFGPU_TC_SPLIT", str(split))
    a, A, b = problem(3, (31, 31, 31), seed=51)
    M = MF3D(A, 31, 31, 31, 1, 4, precision=MFGPU_MIXED)
    M.Factor()
    x = M.Solve(b[0])
    assert relres(A, x, b[0]) <= 2 * TOL
    assert M.stats()["iterations"] <= (12 if split == 1 else 6)
