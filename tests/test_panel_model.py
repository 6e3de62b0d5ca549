"""CPU model of the panel kernels' algorithm (csrc/kernels_panel.cu): the
diagonal block factored right-looking over 32-column blocks with the block
inverses (k_diag_factor), the rows below by blocked substitution with L11 and
those inverses (k_panel_trsm).  The model follows the kernels' order of
operations block by block and must reproduce a dense Cholesky of the panel
(numpy) to rounding, for full and ragged panel widths; it pins the formulas,
the GPU tests pin the kernels against the oracle."""
import numpy as np
import pytest


def diag_factor_model(A11):
    """Returns (L11, [Li_b]) for the kb x kb SPD block, 32-column blocks."""
    kb = A11.shape[0]
    A = np.tril(A11).astype(np.float64).copy()
    Li = []
    for c0 in range(0, kb, 32):
        jb = min(32, kb - c0)
        c1 = c0 + jb
        # warp Cholesky of the diagonal block, four columns at a time
        B = A[c0:c1, c0:c1]
        for jj in range(0, jb, 4):
            for j in range(jj, min(jj + 4, jb)):
                B[j, j] = np.sqrt(B[j, j])
                B[j + 1:, j] /= B[j, j]
                for l in range(j + 1, min(jj + 4, jb)):
                    B[l:, l] -= B[l:, j] * B[l, j]
            hi = min(jj + 4, jb)
            for l in range(hi, jb):                       # rank-4 update to the right
                B[l:, l] -= B[l:, jj:hi] @ B[l, jj:hi]
        A[c0:c1, c0:c1] = np.tril(B)
        # right-looking inverse of the block, lane = column
        X = np.eye(jb)
        Lb = A[c0:c1, c0:c1]
        for t in range(jb):
            X[t, :] /= Lb[t, t]
            X[t + 1:, :] -= np.outer(Lb[t + 1:, t], X[t, :])
        Li.append(np.tril(X))
        if c1 >= kb:
            break
        # rows below the block times that inverse, then the rest of the block
        A[c1:, c0:c1] = A[c1:, c0:c1] @ Li[-1].T
        P = A[c1:, c0:c1]
        A[c1:, c1:] -= np.tril(P @ P.T)
    return np.tril(A), Li


def panel_trsm_model(X, L11, Li):
    """Z = X L11^{-T} by blocked substitution over 32-column blocks."""
    Z = X.astype(np.float64).copy()
    kb = L11.shape[0]
    for b, c0 in enumerate(range(0, kb, 32)):
        c1 = min(c0 + 32, kb)
        Y = Z[:, c0:c1] - Z[:, :c0] @ L11[c0:c1, :c0].T
        Z[:, c0:c1] = Y @ Li[b].T
    return Z


@pytest.mark.parametrize("kb,rows", [(128, 300), (64, 130), (100, 77), (33, 5), (7, 40)])
def test_panel_model_matches_dense_cholesky(kb, rows):
    rng = np.random.default_rng(kb * 1000 + rows)
    M = rng.standard_normal((kb + rows, kb + rows))
    S = M @ M.T + (kb + rows) * np.eye(kb + rows)      # SPD front
    L = np.linalg.cholesky(S)
    L11, Li = diag_factor_model(S[:kb, :kb])
    assert np.allclose(L11, L[:kb, :kb], rtol=1e-12, atol=1e-12 * np.abs(L).max())
    for b, c0 in enumerate(range(0, kb, 32)):
        c1 = min(c0 + 32, kb)
        assert np.allclose(Li[b] @ L11[c0:c1, c0:c1], np.eye(c1 - c0), atol=1e-12)
    L21 = panel_trsm_model(S[kb:, :kb], L11, Li)
    assert np.allclose(L21, L[kb:, :kb], rtol=1e-10, atol=1e-11 * np.abs(L).max())
