"""GPU: separator widths 2 and 3 (the reference fixture's wider stencils,
test_include/DE/buildLaplacian.hpp:18-35), factored by pivoted LU on the GPU,
against the reference itself (oracle/_ref/ref_harness) on the same seeded
variable-coefficient inputs.

With variable coefficients these operators are nonsymmetric (and at width 3
their symmetric part is indefinite), so the reference's partial-pivoting LU
of every pivot block (include/LinAlg/dense.hpp:180-227) is the factorization
to match: kernels_lu.cu pivots among the pivot rows exactly as dgetrf on A22
does.  Tolerances (relative, per right-hand side): solve within 1e-12 of the
reference before and after a localized update, apply within 1e-12, FP64
residual within 1e-12.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import refio
from mfgpu import MF2D, MF3D, MFBatch, MFGPU_MIXED, stencil
from problems import rel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [
    (2, (63, 63), 2, 4, (0.5, 2.0)),
    (2, (30, 27), 3, 5, (0.5, 2.0)),     # ragged, remainder boxes
    (2, (63, 63), 3, 4, (0.1, 10.0)),    # strong contrast
    (3, (15, 15, 15), 2, 4, (0.5, 2.0)),
    (3, (11, 9, 13), 3, 3, (0.5, 2.0)),  # ragged 3D
]


def _make(dim, N, A, w, ms, **kw):
    return (MF2D(A, N[0], N[1], w, ms, **kw) if dim == 2
            else MF3D(A, N[0], N[1], N[2], w, ms, **kw))


@pytest.mark.parametrize("dim,N,w,ms,rng_", CASES)
def test_wide_stencil_factor_update_solve_apply_vs_reference(dim, N, w, ms, rng_):
    if not refio.have_reference():
        pytest.fail("reference harness oracle/_ref/ref_harness is not built")
    lo, hi = rng_
    a1 = stencil.loguniform_coefficients(N, lo, hi, 20261203 + 71, width=w)
    a2 = stencil.scale_box(a1, [2] * dim, 5 if dim == 2 else 3, 10.0, width=w)
    A1 = stencil.build_laplacian(a1, width=w)
    A2 = stencil.build_laplacian(a2, width=w)
    d = A1.to_scipy()
    assert abs(d - d.T).max() > 1e-6 * abs(d).max()          # nonsymmetric
    mod = stencil.modified_dofs(A1, A2)
    b = stencil.uniform_rhs(A1.n, 2, 20261203 + 72)
    with tempfile.TemporaryDirectory() as tmp:
        R = refio.run_reference(tmp, dim, N, w, ms, a1, a2, b, dump_symbolic=0,
                                threads=os.cpu_count() or 1)
    np.testing.assert_array_equal(R["A1.val"], A1.val)          # the same matrix
    assert np.array_equal(np.asarray(R["moddofs"], np.int32), mod)
    F = _make(dim, N, A1, w, ms)
    F.Factor()
    X1, Y1 = F.Solve(b.T), F.Apply(b.T)
    F.Update(A2, mod)
    assert 0 < F.stats()["fronts"] < F.info()["n_fronts"]    # root paths only
    X2, Y2 = F.Solve(b.T), F.Apply(b.T)
    for r in range(b.shape[0]):
        for tag, A, X, Y in (("f1", A1, X1, Y1), ("f2", A2, X2, Y2)):
            fe = rel(X[:, r], R[f"{tag}.solve.{r}"])
            ae = rel(Y[:, r], R[f"{tag}.apply.{r}"])
            res = float(np.linalg.norm(A.matvec(X[:, r]) - b[r]) / np.linalg.norm(b[r]))
            print(f"{dim}D {N} width {w} {tag} rhs {r}: solve vs reference {fe:.2e}, "
                  f"apply {ae:.2e}, residual {res:.2e}")
            assert fe < 1e-12 and ae < 1e-12 and res < 1e-12
    # an update equals a from-scratch LU factorization of the new matrix
    G = _make(dim, N, A2, w, ms)
    G.Factor()
    assert rel(G.Solve(b[0]), X2[:, 0]) < 1e-13


def test_wide_stencils_are_fp64_single_problem_only():
    N, w = (31, 31), 2
    A = stencil.build_laplacian(stencil.loguniform_coefficients(N, 0.5, 2.0, 3, width=w), width=w)
    with pytest.raises(ValueError, match="FP64"):
        MF2D(A, N[0], N[1], w, 4, precision=MFGPU_MIXED)
    with pytest.raises(ValueError, match="width"):
        MFBatch([(A, N, w, 4)])


def test_reference_driver_with_width_2_runs_on_the_gpu_path():
    """The reference's own test driver (test_src/DE/testMF2D.cpp), compiled
    unchanged against the drop-in headers, with separator width 2."""
    exe = os.path.join(ROOT, "oracle", "_ref", "dropin_testMF2D")
    if not os.path.isfile(exe):
        pytest.fail("reference drivers were not built against the drop-in headers")
    p = subprocess.run([exe, "63", "63", "2"], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    import re
    nums = lambda label: [float(x) for x in re.findall(re.escape(label) + r"\s*\n\s*([0-9.eE+-]+)",
                                                       p.stdout)]
    print(p.stdout[-1500:])
    assert nums("Relative apply error is:")[0] < 1e-13
    assert nums("Relative solve error is:")[0] < 1e-12
    assert nums("Relative apply error after updating is:")[0] < 1e-13
