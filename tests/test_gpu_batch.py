"""GPU: batches of independent problems in one handle (mfgpu_batch_create).

Each problem of a batch must give the same solution as its own handle (FP64:
within 1e-13 of it and 1e-12 of the oracle; mixed: every problem and every
right-hand side at relative residual <= 1e-10), and a localized update of one
member must leave the others untouched.
"""
import numpy as np
import pytest

import mf_oracle
from mfgpu import MF2D, MF3D, MFBatch, MFGPU_MIXED, stencil
from problems import patch_update, problem, rel

pytestmark = pytest.mark.gpu

BATCH = [(2, (31, 31), 4), (2, (63, 63), 4), (2, (127, 127), 4), (3, (15, 15, 15), 4),
         (3, (13, 17, 11), 3), (2, (23, 57), 4)]


def single(dim, N, A, ms, **kw):
    return MF2D(A, N[0], N[1], 1, ms, **kw) if dim == 2 else MF3D(A, N[0], N[1], N[2], 1, ms, **kw)


def build(seed0=100):
    probs, rhs = [], []
    for i, (dim, N, ms) in enumerate(BATCH):
        a, A, b = problem(dim, N, seed=seed0 + i, nrhs=1 + i % 3)
        probs.append((a, A, N, ms, dim))
        rhs.append(b.T)
    return probs, rhs


def test_batch_fp64_matches_single_handles_and_oracle():
    probs, rhs = build()
    B = MFBatch([(A, N, 1, ms) for a, A, N, ms, dim in probs])
    B.Factor()
    X = B.split(B.Solve(B.join(rhs)))
    Y = B.split(B.Apply(B.join(rhs)))
    for (a, A, N, ms, dim), b, x, y in zip(probs, rhs, X, Y):
        F = single(dim, N, A, ms)
        F.Factor()
        k = b.shape[1]
        assert rel(x[:, :k], F.Solve(b)) < 1e-13
        assert rel(y[:, :k], F.Apply(b)) < 1e-13
        assert not x[:, k:].any()                  # zero-padded right-hand sides stay zero
        O = mf_oracle.MFOracle(A.to_scipy(), N, 1, ms)
        O.factor()
        assert rel(x[:, 0], O.solve(b[:, 0])) < 1e-12


def test_batch_update_touches_one_member():
    probs, rhs = build(200)
    B = MFBatch([(A, N, 1, ms) for a, A, N, ms, dim in probs])
    B.Factor()
    before = B.split(B.Solve(B.join(rhs)))
    j = 2
    a, A, N, ms, dim = probs[j]
    a2, _ = patch_update(a, N, 9, 10.0, seed=4)
    A2 = stencil.build_laplacian(a2)
    mod = stencil.modified_dofs(A, A2)
    B.Update([A2 if p == j else None for p in range(len(probs))],
             [mod if p == j else [] for p in range(len(probs))])
    st = B.stats()
    assert 0 < st["fronts"] < B.info()["n_fronts"]
    after = B.split(B.Solve(B.join(rhs)))
    for p in range(len(probs)):
        if p != j:
            assert np.array_equal(after[p], before[p])
    G = single(dim, N, A2, ms)
    G.Factor()
    k = rhs[j].shape[1]
    assert rel(after[j][:, :k], G.Solve(rhs[j])) < 1e-13
    assert rel(after[j], before[j]) > 1e-6


def test_batch_mixed_every_problem_reaches_tolerance():
    probs, rhs = build(300)
    B = MFBatch([(A, N, 1, ms) for a, A, N, ms, dim in probs], precision=MFGPU_MIXED)
    B.Factor()
    X = B.split(B.Solve(B.join(rhs)))
    assert B.stats()["residual"] <= 1e-10
    for (a, A, N, ms, dim), b, x in zip(probs, rhs, X):
        for c in range(b.shape[1]):
            r = np.linalg.norm(A.matvec(x[:, c]) - b[:, c]) / np.linalg.norm(b[:, c])
            assert r <= 2e-10
    # each member's refinement is its own: alone it converges to the same answer
    a, A, N, ms, dim = probs[3]
    M = single(dim, N, A, ms, precision=MFGPU_MIXED)
    M.Factor()
    assert rel(X[3][:, :rhs[3].shape[1]], M.Solve(rhs[3])) < 1e-8
