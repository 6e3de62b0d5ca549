"""Seeded test problems shared by the CPU and GPU tests (test helper)."""
import numpy as np

from mfgpu import stencil

SEED0 = 20261203


def problem(dim, N, coef="logu", lo=0.1, hi=10.0, seed=1, nrhs=1):
    """(coefficients, CSR, right-hand sides (nrhs, n))."""
    if coef == "uniform":
        a = stencil.uniform_coefficients(N)
    else:
        a = stencil.loguniform_coefficients(N, lo, hi, SEED0 + seed)
    A = stencil.build_laplacian(a)
    b = stencil.uniform_rhs(A.n, nrhs, SEED0 + 1000 + seed)
    return a, A, b


def patch_update(a, N, side, factor, seed):
    """Coefficients scaled by `factor` on a box of `side` cells at a seeded spot."""
    rng = np.random.Generator(np.random.PCG64(SEED0 + 5000 + seed))
    lo = [int(rng.integers(0, n - side + 1)) for n in N]
    a2 = stencil.scale_box(a, lo, side, factor)
    return a2, lo


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))
