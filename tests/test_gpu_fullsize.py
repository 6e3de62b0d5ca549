"""GPU parity at the full sizes of the measured workloads, against the
reference itself (oracle/_ref/ref_harness: the reference's MF2D compiled from
its own sources, run here on the host) on the same seeded inputs.

* The CPU-runnable configuration exactly as specified: 2D 127^2, a = 1,
  maxSideLength 4, one right-hand side, a 9 x 9-cell patch x10 at a seeded
  position; factor, localized update, solve and apply.
* The 2D 1023^2 configuration at full size: a log-uniform in [0.1, 10],
  maxSideLength 8, four right-hand sides; factor, localized update, solve.
* The mixed-precision path on both, against the same reference solutions.
* The stepped FP64 path (one launch per panel step and kernel) forced on
  levels the cooperative kernel would take.

Tolerances (relative, 2-norm, per right-hand side): FP64 solve within 1e-12 of
the reference and apply within 1e-13; FP64 residuals within 1e-12 (the
reference's own forward error at 1023^2 is about 1.5e-12 against a known
solution, so the bar is the reference's accuracy); mixed residuals within
1e-10 after refinement and mixed solutions within 1e-8 of the reference
(forward error <= condition number x residual; these operators have
condition numbers below 1e3 relative to that bound).  Every figure is printed
(pytest -s).
"""
import os
import sys
import tempfile

import numpy as np
import pytest

import refio
from mfgpu import MF2D, MFGPU_MIXED
from problems import rel

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402  (the workload definitions the measurements use)


def _need_reference():
    if not refio.have_reference():
        pytest.fail("reference harness oracle/_ref/ref_harness is not built")


def _run(workload):
    """Inputs of a bench workload, the reference's records on them, and ours."""
    _need_reference()
    w = bench.WORKLOADS[workload]
    a1, a2, A1, A2, mod, b, lo = bench.make_problem(w)
    with tempfile.TemporaryDirectory() as d:
        R = refio.run_reference(d, 2, w["N"], 1, w["max_side"], a1, a2, b, dump_symbolic=0,
                                threads=os.cpu_count() or 1)
    return w, A1, A2, mod, b, R


def _ours(w, A1, A2, mod, b, **kw):
    N = w["N"]
    F = MF2D(A1, N[0], N[1], 1, w["max_side"], **kw)
    F.Factor()
    X1 = F.Solve(b.T)
    Y1 = None if kw.get("precision") == MFGPU_MIXED else F.Apply(b.T)
    F.Update(A2, mod)
    X2 = F.Solve(b.T)
    Y2 = None if kw.get("precision") == MFGPU_MIXED else F.Apply(b.T)
    F.close()
    return X1, Y1, X2, Y2


def _resid(A, x, b):
    return float(np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b))


def _check_fp64(name, w, A1, A2, mod, b, R):
    assert np.array_equal(np.asarray(R["moddofs"], np.int32), mod)   # same modified DOFs
    X1, Y1, X2, Y2 = _ours(w, A1, A2, mod, b)
    for r in range(b.shape[0]):
        for tag, A, X, Y in (("f1", A1, X1, Y1), ("f2", A2, X2, Y2)):
            xr, yr = R[f"{tag}.solve.{r}"], R[f"{tag}.apply.{r}"]
            fe, ae = rel(X[:, r], xr), rel(Y[:, r], yr)
            ours, theirs = _resid(A, X[:, r], b[r]), float(R[f"{tag}.resid.{r}"][0])
            print(f"{name} {tag} rhs {r}: forward error vs reference {fe:.2e}, apply {ae:.2e}, "
                  f"residual ours {ours:.2e} reference {theirs:.2e}")
            assert fe < 1e-12 and ae < 1e-13 and ours < 1e-12


def _check_mixed(name, w, A1, A2, mod, b, R):
    X1, _, X2, _ = _ours(w, A1, A2, mod, b, precision=MFGPU_MIXED)
    for r in range(b.shape[0]):
        for tag, A, X in (("f1", A1, X1), ("f2", A2, X2)):
            fe = rel(X[:, r], R[f"{tag}.solve.{r}"])
            res = _resid(A, X[:, r], b[r])
            print(f"{name} mixed {tag} rhs {r}: forward error vs reference {fe:.2e}, "
                  f"residual {res:.2e}")
            assert res <= 1e-10 and fe < 1e-8


@pytest.fixture(scope="module")
def cfg0():
    return _run("2d-127")


@pytest.fixture(scope="module")
def cfg1():
    return _run("2d-1023")


def test_cpu_runnable_configuration_exactly_vs_reference(cfg0):
    w, A1, A2, mod, b, R = cfg0
    assert np.all(A1.val[A1.col_ind == np.arange(A1.n).repeat(np.diff(A1.row_ptr))] == 4.0)
    assert len(mod) > 0
    _check_fp64("2d-127", *cfg0)


def test_cpu_runnable_configuration_mixed_vs_reference(cfg0):
    _check_mixed("2d-127", *cfg0)


def test_2d_1023_full_size_vs_reference(cfg1):
    _check_fp64("2d-1023", *cfg1)


def test_2d_1023_full_size_mixed_vs_reference(cfg1):
    _check_mixed("2d-1023", *cfg1)


def test_stepped_factor_path_vs_reference(cfg0, monkeypatch):
    """MFGPU_STEPPED=1: every level the cooperative kernel would take runs as
    per-panel k_potrf / k_trsm / k_syrk launches instead."""
    monkeypatch.setenv("MFGPU_STEPPED", "1")
    w, A1, A2, mod, b, R = cfg0
    N = w["N"]
    F = MF2D(A1, N[0], N[1], 1, w["max_side"])
    F.profile(True)
    F.Factor()
    prof = F.profile_read()
    assert prof["potrf"]["launches"] > 0 and prof["trsm"]["launches"] > 0
    assert prof["syrk"]["launches"] > 0 and prof["coop"]["launches"] == 0
    X = F.Solve(b.T)
    F.Update(A2, mod)
    X2 = F.Solve(b.T)
    F.close()
    for r in range(b.shape[0]):
        e1, e2 = rel(X[:, r], R[f"f1.solve.{r}"]), rel(X2[:, r], R[f"f2.solve.{r}"])
        print(f"2d-127 stepped rhs {r}: forward error vs reference {e1:.2e} / after update {e2:.2e}")
        assert e1 < 1e-12 and e2 < 1e-12
