"""The product's host-side symbolic schedule (csrc/schedule.cpp via the
host-only mfgpu_symbolic_* entry points) against the reference.

* DOF lists of every front and separator equal the reference's (golden).
* The assembly task tables, executed with numpy on the oracle's numbers,
  rebuild every front and separator bit for bit (the extend-add maps).
* A numpy model of the whole algorithm driven by those tables (assembly,
  partial Cholesky, separator sums, solve sweeps) matches the oracle.
* The update marks exactly the root paths of the leaves holding modified DOFs,
  a subset of what the reference refactors.
"""
import numpy as np
import pytest
import scipy.linalg as sla

import golden_cases as gc
import mf_oracle
import taskemu
from mfgpu import Symbolic, stencil


@pytest.mark.parametrize("name", gc.NAMES)
def test_dof_lists_match_reference(name, lib):
    case, a1, a2, rhs, G = gc.load(name)
    S = Symbolic(case["dim"], case["N"], 1, case["ms"])
    assert S.levels == int(G["levels"])
    f = 0
    for ell in range(S.levels):
        ints, bds = gc.unflatten(G, f"box_{ell}_int"), gc.unflatten(G, f"box_{ell}_bd")
        for b in range(len(ints)):
            F = S.front(f)
            f += 1
            assert (F["level"], F["box"]) == (ell, b)
            assert np.array_equal(F["dofs"][:F["n"]], ints[b])
            assert np.array_equal(F["dofs"][F["n"]:], bds[b])
    k = 0
    for ell in range(1, S.levels):
        for e, dofs in enumerate(gc.unflatten(G, f"sep_{ell}")):
            s = S.sep(k)
            k += 1
            assert (s["level"], s["idx"]) == (ell, e)
            assert np.array_equal(s["dofs"], dofs)


def _um(box, sizes):
    U = box.A11post.copy()
    p = 0
    for sz in sizes:
        U[p:p + sz, p:p + sz] = box.S[p:p + sz, p:p + sz]
        p += sz
    return U


@pytest.mark.parametrize("dim,N,ms", [(2, (31, 31), 4), (2, (23, 57), 4), (3, (15, 15, 15), 4),
                                      (3, (13, 17, 11), 3)])
def test_assembly_tasks_rebuild_fronts_bit_for_bit(dim, N, ms, lib):
    A = stencil.build_laplacian(stencil.loguniform_coefficients(N, 0.1, 10.0, 3)).to_scipy()
    O = mf_oracle.MFOracle(A, N, 1, ms, symmetric_schur=True)
    O.factor()
    S = Symbolic(dim, N, 1, ms)
    E = taskemu.Emu(S, A)
    L = S.levels
    for f, F in enumerate(E.fronts):
        if F["level"] == 0:
            continue
        box = O.boxes[F["level"]][F["box"]]
        sizes = [len(O.seps[F["level"]][e].dofs) for e in O._nbor_seps(F["box"], F["level"]) if e != -1]
        M = np.zeros((F["n"] + F["m"],) * 2)
        M[F["n"]:, F["n"]:] = _um(box, sizes)
        E.set_block(f, M)
    for k, s in enumerate(E.seps):
        E.set_sep(k, O.seps[s["level"]][s["idx"]].A11)
    saved = E.F.copy()
    for f, F in enumerate(E.fronts):
        ell, b, n = F["level"], F["box"], F["n"]
        E.F[:] = saved
        E.run(E.ftasks, [f])
        M = E.block(f)
        box = O.boxes[ell][b]
        assert np.array_equal(np.tril(M[:n, :n]), np.tril(box.A22))
        if ell == 0:
            continue
        if ell == L - 1:
            A12 = A[np.asarray(box.bd)][:, np.asarray(box.int)].toarray()
            A11 = A[np.asarray(box.bd)][:, np.asarray(box.bd)].toarray()
        else:
            A12, A11 = box.A12_asm, box.A11_asm
        assert np.array_equal(M[n:, :n], A12)
        B, R = M[n:, n:].copy(), A11.copy()
        p = 0
        for e in O._nbor_seps(b, ell):
            if e == -1:
                continue
            sz = len(O.seps[ell][e].dofs)
            assert not B[p:p + sz, p:p + sz].any()      # separator diagonal blocks start at zero
            B[p:p + sz, p:p + sz] = 0
            R[p:p + sz, p:p + sz] = 0
            p += sz
        assert np.array_equal(np.tril(B), np.tril(R))
    E.F[:] = saved
    for k, s in enumerate(E.seps):
        sp = O.seps[s["level"]][s["idx"]]
        E.run(E.stasks, [k])
        assert np.array_equal(np.tril(E.sep_block(k)), np.tril(sp.A11_base))
        E.run(E.atasks, [k])
        assert np.array_equal(np.tril(E.sep_block(k)), np.tril(sp.A11))


def _model_solve(S, E, b):
    """Algorithm model: tasks + partial Cholesky + solve sweeps (numpy)."""
    for ell in range(S.levels - 1, -1, -1):
        fl, sl = E.level_fronts(ell), E.level_seps(ell)
        E.run(E.stasks, sl)
        E.run(E.ftasks, fl)
        for f in fl:
            n = E.fronts[f]["n"]
            M = E.block(f)
            L11 = np.linalg.cholesky(M[:n, :n])
            L21 = sla.solve_triangular(L11, M[n:, :n].T, lower=True).T
            M[:n, :n], M[n:, :n] = L11, L21
            M[n:, n:] -= L21 @ L21.T
            E.set_block(f, M)
        E.run(E.atasks[0::2], sl)
        E.run(E.atasks[1::2], sl)
    X, W, Fr = b.copy(), {}, E.fronts
    for ell in range(S.levels - 1, 0, -1):
        for f in E.level_fronts(ell):
            n, d, M = Fr[f]["n"], Fr[f]["dofs"], np.tril(E.block(f))
            y = sla.solve_triangular(M[:n, :n], X[d[:n]], lower=True)
            X[d[:n]] = y
            W[f] = -(M[n:, :n] @ y)
        for k in E.level_seps(ell):
            s = E.seps[k]
            (b0, b1), (r0, r1) = s["boxes"], s["rows"]
            d, n0, n1 = s["dofs"], Fr[b0]["n"], Fr[b1]["n"]
            X[d] = (X[d] + W[b0][r0 - n0:r0 - n0 + len(d)]) + W[b1][r1 - n1:r1 - n1 + len(d)]
    M, d = np.tril(E.block(0)), Fr[0]["dofs"]
    X[d] = sla.solve_triangular(M, sla.solve_triangular(M, X[d], lower=True), lower=True, trans=1)
    for ell in range(1, S.levels):
        for f in E.level_fronts(ell):
            n, d, M = Fr[f]["n"], Fr[f]["dofs"], np.tril(E.block(f))
            X[d[:n]] = sla.solve_triangular(M[:n, :n], X[d[:n]] - M[n:, :n].T @ X[d[n:]],
                                            lower=True, trans=1)
    return X


@pytest.mark.parametrize("dim,N,ms", [(2, (31, 31), 4), (3, (13, 17, 11), 3)])
def test_algorithm_model_matches_oracle(dim, N, ms, lib):
    A = stencil.build_laplacian(stencil.loguniform_coefficients(N, 0.1, 10.0, 5)).to_scipy()
    b = stencil.uniform_rhs(A.shape[0], 1, 9)[0]
    S = Symbolic(dim, N, 1, ms)
    x = _model_solve(S, taskemu.Emu(S, A), b)
    O = mf_oracle.MFOracle(A, N, 1, ms)
    O.factor()
    xo = O.solve(b)
    assert np.linalg.norm(x - xo) <= 1e-13 * np.linalg.norm(xo)


@pytest.mark.parametrize("dim,N,w,ms", [(2, (31, 31), 2, 4), (2, (30, 27), 3, 5),
                                        (3, (11, 9, 13), 2, 3), (3, (15, 15, 15), 3, 4)])
def test_algorithm_model_wide_stencils(dim, N, w, ms, lib):
    """Separator widths 2 and 3: with uniform coefficients the fixture's wider
    stencils are symmetric positive definite, and the schedule's task tables
    executed with partial Cholesky solve them as the oracle does."""
    A = stencil.build_laplacian(stencil.uniform_coefficients(N, w), width=w).to_scipy()
    assert (A - A.T).nnz == 0
    b = stencil.uniform_rhs(A.shape[0], 1, 9)[0]
    S = Symbolic(dim, N, w, ms)
    x = _model_solve(S, taskemu.Emu(S, A), b)
    O = mf_oracle.MFOracle(A, N, w, ms)
    O.factor()
    xo = O.solve(b)
    assert np.linalg.norm(x - xo) <= 1e-13 * np.linalg.norm(xo)


def _model_solve_lu(S, E, b):
    """Algorithm model for nonsymmetric matrices: full-storage tables + partial
    LU with row pivoting inside each pivot block + solve sweeps (numpy)."""
    fac = {}
    for ell in range(S.levels - 1, -1, -1):
        fl, sl = E.level_fronts(ell), E.level_seps(ell)
        E.run(E.stasks, sl)
        E.run(E.ftasks, fl)
        for f in fl:
            n = E.fronts[f]["n"]
            M = E.block_full(f)
            lu, piv = sla.lu_factor(M[:n, :n])
            U = np.triu(lu)
            L = np.tril(lu, -1) + np.eye(n)
            M12 = M[:n, n:].copy()
            for i, p in enumerate(piv):               # the row swaps of the pivot block
                M12[[i, p]] = M12[[p, i]]
            L21 = sla.solve_triangular(U, M[n:, :n].T, trans=1, lower=False).T
            U12 = sla.solve_triangular(L, M12, lower=True, unit_diagonal=True)
            M[n:, n:] -= L21 @ U12
            E.set_block_full(f, M)
            fac[f] = (lu, piv, L21, U12)
        E.run(E.atasks[0::2], sl)
        E.run(E.atasks[1::2], sl)
    X, W, Fr = b.copy(), {}, E.fronts
    for ell in range(S.levels - 1, 0, -1):
        for f in E.level_fronts(ell):
            n, d = Fr[f]["n"], Fr[f]["dofs"]
            lu, piv, L21, U12 = fac[f]
            y = X[d[:n]].copy()
            for i, p in enumerate(piv):
                y[[i, p]] = y[[p, i]]
            y = sla.solve_triangular(lu, y, lower=True, unit_diagonal=True)
            X[d[:n]] = y
            W[f] = -(L21 @ y)
        for k in E.level_seps(ell):
            s = E.seps[k]
            (b0, b1), (r0, r1) = s["boxes"], s["rows"]
            d, n0, n1 = s["dofs"], Fr[b0]["n"], Fr[b1]["n"]
            X[d] = (X[d] + W[b0][r0 - n0:r0 - n0 + len(d)]) + W[b1][r1 - n1:r1 - n1 + len(d)]
    d = Fr[0]["dofs"]
    X[d] = sla.lu_solve(fac[0][:2], X[d])
    for ell in range(1, S.levels):
        for f in E.level_fronts(ell):
            n, d = Fr[f]["n"], Fr[f]["dofs"]
            lu, piv, L21, U12 = fac[f]
            X[d[:n]] = sla.solve_triangular(lu, X[d[:n]] - U12 @ X[d[n:]], lower=False)
    return X


@pytest.mark.parametrize("dim,N,w,ms", [(2, (31, 31), 2, 4), (2, (30, 27), 3, 5),
                                        (3, (11, 9, 13), 2, 3), (3, (15, 15, 15), 3, 4),
                                        (2, (31, 31), 1, 4)])
def test_full_storage_tables_solve_nonsymmetric_stencils(dim, N, w, ms, lib):
    """Variable coefficients make the fixture's width-2/3 stencils
    nonsymmetric: the full-storage task tables executed with pivoted partial
    LU (the reference's factorization) solve them as the oracle does."""
    a = stencil.loguniform_coefficients(N, 0.5, 2.0, 5, width=w)
    A = stencil.build_laplacian(a, width=w).to_scipy()
    if w > 1:
        assert abs(A - A.T).max() > 1e-6 * abs(A).max()
    b = stencil.uniform_rhs(A.shape[0], 1, 9)[0]
    S = Symbolic(dim, N, w, ms, full=True)
    x = _model_solve_lu(S, taskemu.Emu(S, A), b)
    O = mf_oracle.MFOracle(A, N, w, ms)
    O.factor()
    xo = O.solve(b)
    assert np.linalg.norm(x - xo) <= 1e-12 * np.linalg.norm(xo)
    assert np.linalg.norm(A @ x - b) <= 1e-12 * np.linalg.norm(b)


@pytest.mark.parametrize("dim,N,ms,side", [(2, (127, 127), 4, 9), (3, (23, 23, 23), 4, 4)])
def test_update_marks_root_paths(dim, N, ms, side, lib):
    a = stencil.loguniform_coefficients(N, 0.1, 10.0, 8)
    a2 = stencil.scale_box(a, [3] * dim, side, 10.0)
    A1, A2 = stencil.build_laplacian(a), stencil.build_laplacian(a2)
    mod = stencil.modified_dofs(A1, A2)
    S = Symbolic(dim, N, 1, ms)
    dirty, _ = S.dirty(mod)
    fronts = [S.front(f) for f in range(S.n_fronts)]
    # leaves holding a modified DOF (the reference's marking, src/DE/mf2d.cpp:163-174)
    O = mf_oracle.MFOracle(A1.to_scipy(), N, 1, ms)
    O.factor()
    O.marked_boxes, O.marked_seps = set(), set()
    leaves = set()
    bps = 1 << (O.levels - 1)
    for d in mod:
        c = [d % N[0], (d // N[0]) % N[1]] + ([d // (N[0] * N[1])] if dim == 3 else [])
        q = [min(c[x] // (O.bw[x] + 1), bps - 1) for x in range(dim)]
        leaves.add(q[0] + q[1] * bps + (q[2] * bps * bps if dim == 3 else 0))
    expect = set()
    for b in leaves:
        ell = O.levels - 1
        while True:
            expect.add((ell, b))
            if ell == 0:
                break
            b = O._parent(b, ell)
            ell -= 1
    got = {(F["level"], F["box"]) for F, dflag in zip(fronts, dirty) if dflag}
    assert got == expect
    # the reference refactors a superset: parents of both boxes of every marked separator
    ref = set()
    O.marked_boxes = set(leaves)
    for ell in range(O.levels - 1, 0, -1):
        ref |= {(ell, b) for b in O.marked_boxes}
        seps = set()
        for b in O.marked_boxes:
            seps.update(e for e in O._nbor_seps(b, ell) if e != -1)
        O.marked_boxes = {O._parent(bx, ell) for e in seps for bx in O._nbor_boxes(e, ell)}
    ref |= {(0, 0)}
    assert got <= ref


def _model_solve_forest(S, E, b):
    """Algorithm model for a batch: every level, roots included, through the
    generic forward sweep, then the generic backward sweep."""
    for ell in range(S.levels - 1, -1, -1):
        fl, sl = E.level_fronts(ell), E.level_seps(ell)
        E.run(E.stasks, sl)
        E.run(E.ftasks, fl)
        for f in fl:
            n = E.fronts[f]["n"]
            M = E.block(f)
            L11 = np.linalg.cholesky(M[:n, :n])
            L21 = sla.solve_triangular(L11, M[n:, :n].T, lower=True).T
            M[:n, :n], M[n:, :n] = L11, L21
            M[n:, n:] -= L21 @ L21.T
            E.set_block(f, M)
        E.run(E.atasks[0::2], sl)
        E.run(E.atasks[1::2], sl)
    X, W, Fr = b.copy(), {}, E.fronts
    for ell in range(S.levels - 1, -1, -1):
        for f in E.level_fronts(ell):
            n, d, M = Fr[f]["n"], Fr[f]["dofs"], np.tril(E.block(f))
            y = sla.solve_triangular(M[:n, :n], X[d[:n]], lower=True)
            X[d[:n]] = y
            W[f] = -(M[n:, :n] @ y)
        for k in E.level_seps(ell):
            s = E.seps[k]
            (b0, b1), (r0, r1) = s["boxes"], s["rows"]
            d, n0, n1 = s["dofs"], Fr[b0]["n"], Fr[b1]["n"]
            X[d] = (X[d] + W[b0][r0 - n0:r0 - n0 + len(d)]) + W[b1][r1 - n1:r1 - n1 + len(d)]
    for ell in range(0, S.levels):
        for f in E.level_fronts(ell):
            n, d, M = Fr[f]["n"], Fr[f]["dofs"], np.tril(E.block(f))
            X[d[:n]] = sla.solve_triangular(M[:n, :n], X[d[:n]] - M[n:, :n].T @ X[d[n:]],
                                            lower=True, trans=1)
    return X


def test_batch_forest_model_matches_oracle(lib):
    # three problems of different depth and dimension in one forest schedule:
    # levels aligned at the leaves, fronts renumbered, DOFs shifted
    import scipy.sparse as sp
    batch = [(2, (31, 31), 1, 4), (2, (63, 63), 1, 4), (3, (13, 17, 11), 1, 3)]
    mats, rhs, xs = [], [], []
    for i, (dim, N, w, ms) in enumerate(batch):
        A = stencil.build_laplacian(stencil.loguniform_coefficients(N, 0.1, 10.0, 20 + i)).to_scipy()
        b = stencil.uniform_rhs(A.shape[0], 1, 30 + i)[0]
        O = mf_oracle.MFOracle(A, N, w, ms)
        O.factor()
        mats.append(A)
        rhs.append(b)
        xs.append(O.solve(b))
    S = Symbolic(0, (0, 0), batch=batch)
    singles = [Symbolic(dim, N, w, ms) for dim, N, w, ms in batch]
    assert S.levels == max(q.levels for q in singles)
    assert S.n_fronts == sum(q.n_fronts for q in singles)
    assert S.ndof == sum(q.ndof for q in singles)
    x = _model_solve_forest(S, taskemu.Emu(S, sp.block_diag(mats, format="csr")),
                            np.concatenate(rhs))
    off = 0
    for b, xo in zip(rhs, xs):
        assert np.linalg.norm(x[off:off + len(b)] - xo) <= 1e-13 * np.linalg.norm(xo)
        off += len(b)
    # dirty marking stays inside the touched problem
    dirty, _ = S.dirty([singles[0].ndof + 5])
    fronts = [S.front(f) for f in range(S.n_fronts)]
    lo, hi = singles[0].ndof, singles[0].ndof + singles[1].ndof
    assert dirty.any()
    for f in np.flatnonzero(dirty):
        d = fronts[f]["dofs"]
        assert len(d) == 0 or (lo <= d.min() and d.max() < hi)
