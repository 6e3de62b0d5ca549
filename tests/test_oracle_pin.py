"""The oracle (oracle/mf_oracle.py) pinned to the reference.

Golden fixtures in tests/golden/ were produced by the reference itself
(tests/golden/make_golden.py runs oracle/_ref/ref_harness, compiled from the
reference sources).  The oracle must reproduce its CSR bit for bit, every
per-level DOF list exactly, and its solve / apply / update results to rounding.
Where the harness is built, a live comparison of per-front blocks runs too.
"""
import hashlib

import numpy as np
import pytest

import golden_cases as gc
import mf_oracle
import refio
from mfgpu import stencil


def _hash(A):
    h = hashlib.sha256()
    for a in (A.row_ptr, A.col_ind, A.val):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", gc.NAMES)
def test_oracle_matches_reference_fixture(name):
    case, a1, a2, rhs, G = gc.load(name)
    A1 = stencil.build_laplacian(a1)
    assert _hash(A1) == str(G["csr_sha256"])           # bit-identical CSR
    O = mf_oracle.MFOracle(A1.to_scipy(), case["N"], 1, case["ms"])
    O.factor()
    assert O.levels == int(G["levels"])
    for ell in range(O.levels):
        ints = gc.unflatten(G, f"box_{ell}_int")
        bds = gc.unflatten(G, f"box_{ell}_bd")
        assert len(ints) == len(O.boxes[ell])
        for b, box in enumerate(O.boxes[ell]):
            assert np.array_equal(box.int, ints[b])
            assert np.array_equal(box.bd, bds[b])
        if ell >= 1:
            seps = gc.unflatten(G, f"sep_{ell}")
            for e, sp in enumerate(O.seps[ell]):
                assert np.array_equal(sp.dofs, seps[e])
    x = O.solve(rhs[0])
    y = O.apply(rhs[0])
    assert np.linalg.norm(x - G["solve"]) <= 1e-13 * np.linalg.norm(G["solve"])
    assert np.linalg.norm(y - G["apply"]) <= 1e-14 * np.linalg.norm(G["apply"])
    if case.get("fronts"):
        for ell in range(1, O.levels):
            for b, box in enumerate(O.boxes[ell]):
                S, P = G[f"S_{ell}_{b}"], G[f"A11post_{ell}_{b}"]
                assert np.abs(box.S - S).max() <= 1e-12 * max(1.0, np.abs(S).max())
                assert np.abs(box.A11post - P).max() <= 1e-12 * max(1.0, np.abs(P).max())
    A2 = stencil.build_laplacian(a2)
    mod = stencil.modified_dofs(A1, A2)
    assert np.array_equal(mod, G["moddofs"])           # the reference's CSR diff
    O.update(A2.to_scipy(), mod)
    xu = O.solve(rhs[0])
    assert np.linalg.norm(xu - G["upd_solve"]) <= 1e-13 * np.linalg.norm(G["upd_solve"])


def test_stencil_builder_widths_and_symmetry(tmp_path):
    # width 1 (5/7-point): bitwise symmetric; the reference's wider stencils
    # (width 2, 3) average faces asymmetrically, and we only match them.
    for N in [(9, 7), (5, 6, 4)]:
        a = stencil.loguniform_coefficients(N, 0.5, 2.0, 3, width=1)
        A = stencil.build_laplacian(a, width=1).to_scipy()
        assert (A - A.T).nnz == 0
    if refio.have_reference():
        for N in [(9, 11), (6, 5, 7)]:
            for w in (1, 2, 3):
                a = stencil.loguniform_coefficients(N, 0.5, 2.0, 4, width=w)
                B = stencil.build_laplacian(a, width=w)
                R = refio.reference_csr(str(tmp_path), len(N), N, w, a)
                assert np.array_equal(R["A1.row_ptr"], B.row_ptr)
                assert np.array_equal(R["A1.col_ind"], B.col_ind)
                assert np.array_equal(R["A1.val"], B.val)


@pytest.mark.skipif(not refio.have_reference(), reason="reference harness not built")
def test_live_reference_front_blocks(tmp_path):
    N, ms = (19, 23), 4
    a = stencil.loguniform_coefficients(N, 0.1, 10.0, 77)
    A = stencil.build_laplacian(a)
    R = refio.run_reference(str(tmp_path), 2, N, 1, ms, a, None, None, dump_fronts=1)
    O = mf_oracle.MFOracle(A.to_scipy(), N, 1, ms)
    O.factor()
    for ell in range(O.levels):
        for b, box in enumerate(O.boxes[ell]):
            p = f"box.{ell}.{b}."
            for nm, v in (("A22", box.A22), ("S", box.S), ("A11post", box.A11post)):
                if v is None or R[p + nm].size == 0:
                    continue
                assert np.abs(R[p + nm] - v).max() <= 1e-12 * max(1.0, np.abs(v).max())


WIDE_CASES = [(2, (23, 19), 2, 4), (2, (30, 27), 3, 5), (2, (64, 40), 2, 6),
              (3, (11, 9, 13), 2, 3), (3, (15, 15, 15), 3, 4)]


@pytest.mark.skipif(not refio.have_reference(), reason="reference harness not built")
@pytest.mark.parametrize("dim,N,w,ms", WIDE_CASES)
def test_wide_stencils_oracle_and_schedule_match_reference(dim, N, w, ms, tmp_path):
    """Separator widths 2 and 3 (the fixture's 9-/13-point 2D and 13-/19-point
    3D stencils): the oracle's DOF lists and solution, and the C++ schedule's
    DOF lists, against the reference run live on the same inputs."""
    from mfgpu import Symbolic
    a = stencil.loguniform_coefficients(N, 0.5, 2.0, 11, width=w)
    A = stencil.build_laplacian(a, width=w)
    rhs = np.random.default_rng(3).uniform(-1, 1, (1, A.n))
    R = refio.run_reference(str(tmp_path), dim, N, w, ms, a, None, rhs)
    L = int(R["levels"][0])
    O = mf_oracle.MFOracle(A.to_scipy(), N, w, ms)
    O.factor()
    S = Symbolic(dim, N, w, ms)
    assert O.levels == L and S.levels == L
    f = k = 0
    for ell in range(L):
        nb = len([x for x in R if x.startswith(f"box.{ell}.") and x.endswith(".int")])
        assert len(O.boxes[ell]) == nb
        for b in range(nb):
            ints, bds = R[f"box.{ell}.{b}.int"], R[f"box.{ell}.{b}.bd"]
            assert np.array_equal(O.boxes[ell][b].int, ints) and np.array_equal(O.boxes[ell][b].bd, bds)
            F = S.front(f)
            f += 1
            assert (F["level"], F["box"]) == (ell, b)
            assert np.array_equal(F["dofs"][:F["n"]], ints) and np.array_equal(F["dofs"][F["n"]:], bds)
        if ell >= 1:
            ns = len([x for x in R if x.startswith(f"sep.{ell}.") and x.endswith(".dofs")])
            for e in range(ns):
                dofs = R[f"sep.{ell}.{e}.dofs"]
                assert np.array_equal(O.seps[ell][e].dofs, dofs)
                s = S.sep(k)
                k += 1
                assert (s["level"], s["idx"]) == (ell, e) and np.array_equal(s["dofs"], dofs)
    x, xr = O.solve(rhs[0]), R["f1.solve.0"]
    assert np.linalg.norm(x - xr) <= 1e-13 * np.linalg.norm(xr)
