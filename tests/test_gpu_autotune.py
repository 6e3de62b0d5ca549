"""GPU: the autotuner (mfgpu_autotune).

The autotuning factorization times every eligible kernel of each level on
freshly assembled fronts and keeps the fastest.  Its result must be a valid
factorization (FP64: the solution within 1e-12 of the size-rule
factorization's, which may use other kernels and so round differently; mixed:
refinement to 1e-10), later full factorizations with the chosen table must
reproduce it bit for bit, and a localized update afterwards must agree with
the size-rule handle's update.
"""
import numpy as np
import pytest

from mfgpu import MF2D, MF3D, MFGPU_MIXED, stencil
from problems import patch_update, problem, rel

pytestmark = pytest.mark.gpu


def make(N, A, **kw):
    return MF2D(A, N[0], N[1], 1, 4, **kw) if len(N) == 2 else MF3D(A, N[0], N[1], N[2], 1, 4, **kw)


def relres(A, x, b):
    return float(np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("N,precision", [((127, 127), None), ((15, 15, 15), None),
                                         ((127, 127), MFGPU_MIXED), ((31, 31, 31), MFGPU_MIXED)])
def test_autotuned_factorization(N, precision):
    kw = {} if precision is None else {"precision": precision}
    a, A, b = problem(len(N), N, seed=71)
    F = make(N, A, **kw)
    choices = F.autotune(2)
    assert len(choices) == F.info()["levels"]
    assert set(choices) <= {"fused", "coop", "tc", "stepped", "panel", "none"}
    G = make(N, A, **kw)                      # size rules
    G.Factor()
    x, y = F.Solve(b[0]), G.Solve(b[0])
    if precision is None:
        assert rel(x, y) < 1e-12
    else:
        assert relres(A, x, b[0]) <= 1e-10
    F.Factor()                                # the tuned table, reused
    assert np.array_equal(F.Solve(b[0]), x)
    a2, _ = patch_update(a, N, 5 if len(N) == 2 else 3, 10.0, seed=9)
    A2 = stencil.build_laplacian(a2)
    mod = stencil.modified_dofs(A, A2)
    F.Update(A2, mod)
    G.Update(A2, mod)
    xu, yu = F.Solve(b[0]), G.Solve(b[0])
    if precision is None:
        assert rel(xu, yu) < 1e-12
    else:
        assert relres(A2, xu, b[0]) <= 1e-10
