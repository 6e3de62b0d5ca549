"""ORACLE — test infrastructure only.

A CPU restatement, in numpy/scipy, of the reference's multifrontal factor /
update / solve / apply path (victorminden/updating-multifrontal).  Only tests,
`__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` may use it, and
only as the checker.  It is pinned against the reference itself: the reference
is compiled from its own sources into oracle/_ref/ref_harness (oracle/Makefile)
and tests/test_oracle_pin.py compares DOF lists, per-front blocks and solutions
of both on the same seeded inputs; tests/golden/ keeps fixtures made by the
reference (tests/golden/make_golden.py).

Each method cites the reference function it restates.  Dense blocks are
column-major in the reference; here they are numpy arrays with the same (row,
column) meaning.  LU with partial pivoting uses scipy (LAPACK dgetrf/dgetrs),
the same routines the reference calls through include/LinAlg/dense.hpp:180-227.
"""
import math

import numpy as np
import scipy.linalg as sla

# ----------------------------------------------------------------------------
# Tree topology, 2D (src/DE/tree2d_common.cpp)
# ----------------------------------------------------------------------------
L2R, T2B = 0, 1


def edge_type(e, ell):                                     # tree2d_common.cpp:8-11
    bps = 1 << ell
    return T2B if (e % (2 * bps - 1)) < bps - 1 else L2R


def edge_idx(row, col, ell, typ):                          # tree2d_common.cpp:15-26
    bps = 1 << ell
    if typ == L2R:
        return row * (2 * bps - 1) + col + bps - 1
    return row * (2 * bps - 1) + col


def edge_coords(e, ell):                                   # tree2d_common.cpp:28-35
    bps = 1 << ell
    if edge_type(e, ell) == L2R:
        e -= bps - 1
    w = 2 * bps - 1
    return e % w, e // w          # (x, y)


def box_coords2(b, bps):
    return b % bps, b // bps


def nbor_edges_of_box(b, ell):                             # tree2d_common.cpp:135-184
    bps = 1 << ell
    x, y = box_coords2(b, bps)
    out = []
    out.append(edge_idx(y, x - 1, ell, T2B) if x > 0 else -1)
    out.append(edge_idx(y, x, ell, T2B) if x < bps - 1 else -1)
    out.append(edge_idx(y - 1, x, ell, L2R) if y > 0 else -1)
    out.append(edge_idx(y, x, ell, L2R) if y < bps - 1 else -1)
    return out


def nbor_boxes_of_edge(e, ell):                            # tree2d_common.cpp:186-211
    bps = 1 << ell
    x, y = edge_coords(e, ell)
    if edge_type(e, ell) == T2B:
        return [x + y * bps, (x + 1) + y * bps]
    return [x + y * bps, x + (y + 1) * bps]


def child_edges(e, ell):                                   # tree2d_common.cpp:91-119
    x, y = edge_coords(e, ell)
    if edge_type(e, ell) == L2R:
        return [edge_idx(2 * y + 1, 2 * x, ell + 1, L2R), edge_idx(2 * y + 1, 2 * x + 1, ell + 1, L2R)]
    return [edge_idx(2 * y, 2 * x + 1, ell + 1, T2B), edge_idx(2 * y + 1, 2 * x + 1, ell + 1, T2B)]


def child_boxes2(b, ell):                                  # tree2d_common.cpp:121-131
    bps = 1 << ell
    x, y = box_coords2(b, bps)
    c = 2 * bps
    return [2 * x + 2 * y * c, 2 * x + (2 * y + 1) * c, (2 * x + 1) + 2 * y * c, (2 * x + 1) + (2 * y + 1) * c]


def parent_box2(b, ell):                                   # tree2d_common.cpp:84-89
    bps = 1 << ell
    x, y = box_coords2(b, bps)
    return x // 2 + (y // 2) * (bps // 2)


def _edge_children_of_box(b, ell, parity):                 # tree2d_common.cpp:37-79
    s = set()
    for c in child_boxes2(b, ell):
        for e in nbor_edges_of_box(c, ell + 1):
            if e == -1:
                continue
            x, y = edge_coords(e, ell + 1)
            t = edge_type(e, ell + 1)
            if (t == T2B and x % 2 == parity) or (t == L2R and y % 2 == parity):
                s.add(e)
    return sorted(s)


def self_edge_children(b, ell):
    return _edge_children_of_box(b, ell, 0)


def shared_edge_children(b, ell):
    return _edge_children_of_box(b, ell, 1)


# ----------------------------------------------------------------------------
# Tree topology, 3D (src/DE/tree3d_common.cpp)
# ----------------------------------------------------------------------------
XN, YN, ZN = 0, 1, 2


def face_type(f, ell):                                     # tree3d_common.cpp:9-19
    bps = 1 << ell
    fps = 2 * (bps - 1) * bps + bps * bps
    f %= fps
    if f >= 2 * (bps - 1) * bps:
        return ZN
    f %= 2 * bps - 1
    return XN if f < bps - 1 else YN


def face_idx(row, col, sli, ell, typ):                     # tree3d_common.cpp:23-40
    bps = 1 << ell
    fps = 2 * (bps - 1) * bps + bps * bps
    if typ == XN:
        return sli * fps + row * (2 * bps - 1) + col
    if typ == YN:
        return sli * fps + row * (2 * bps - 1) + col + bps - 1
    return sli * fps + row * bps + col + 2 * (bps - 1) * bps


def face_coords(f, ell):                                   # tree3d_common.cpp:43-71
    bps = 1 << ell
    fps = 2 * (bps - 1) * bps + bps * bps
    t = face_type(f, ell)
    if t == ZN:
        f -= 2 * (bps - 1) * bps
        z = f // fps
        f -= z * fps
        y = f // bps
        f -= y * bps
        return f, y, z
    if t == YN:
        f -= bps - 1
    z = f // fps
    f -= z * fps
    y = f // (2 * bps - 1)
    f -= y * (2 * bps - 1)
    return f, y, z


def box_coords3(b, bps):
    x = b % bps
    b //= bps
    return x, b % bps, b // bps


def box_lin3(x, y, z, bps):
    return x + y * bps + z * bps * bps


def nbor_faces_of_box(b, ell):                             # tree3d_common.cpp:185-275
    bps = 1 << ell
    x, y, z = box_coords3(b, bps)
    return [face_idx(y, x - 1, z, ell, XN) if x > 0 else -1,
            face_idx(y, x, z, ell, XN) if x < bps - 1 else -1,
            face_idx(y - 1, x, z, ell, YN) if y > 0 else -1,
            face_idx(y, x, z, ell, YN) if y < bps - 1 else -1,
            face_idx(y, x, z - 1, ell, ZN) if z > 0 else -1,
            face_idx(y, x, z, ell, ZN) if z < bps - 1 else -1]


def nbor_boxes_of_face(f, ell):                            # tree3d_common.cpp:277-312
    bps = 1 << ell
    x, y, z = face_coords(f, ell)
    t = face_type(f, ell)
    if t == XN:
        return [box_lin3(x, y, z, bps), box_lin3(x + 1, y, z, bps)]
    if t == YN:
        return [box_lin3(x, y, z, bps), box_lin3(x, y + 1, z, bps)]
    return [box_lin3(x, y, z, bps), box_lin3(x, y, z + 1, bps)]


def child_faces(f, ell):                                   # tree3d_common.cpp:127-164
    x, y, z = face_coords(f, ell)
    row, col, sl = y, x, z
    t = face_type(f, ell)
    if t == XN:
        return [face_idx(2 * row, 2 * col + 1, 2 * sl, ell + 1, XN),
                face_idx(2 * row, 2 * col + 1, 2 * sl + 1, ell + 1, XN),
                face_idx(2 * row + 1, 2 * col + 1, 2 * sl, ell + 1, XN),
                face_idx(2 * row + 1, 2 * col + 1, 2 * sl + 1, ell + 1, XN)]
    if t == YN:
        return [face_idx(2 * row + 1, 2 * col, 2 * sl, ell + 1, YN),
                face_idx(2 * row + 1, 2 * col, 2 * sl + 1, ell + 1, YN),
                face_idx(2 * row + 1, 2 * col + 1, 2 * sl, ell + 1, YN),
                face_idx(2 * row + 1, 2 * col + 1, 2 * sl + 1, ell + 1, YN)]
    return [face_idx(2 * row, 2 * col, 2 * sl + 1, ell + 1, ZN),
            face_idx(2 * row + 1, 2 * col, 2 * sl + 1, ell + 1, ZN),
            face_idx(2 * row, 2 * col + 1, 2 * sl + 1, ell + 1, ZN),
            face_idx(2 * row + 1, 2 * col + 1, 2 * sl + 1, ell + 1, ZN)]


def child_boxes3(b, ell):                                  # tree3d_common.cpp:166-181
    bps = 1 << ell
    x, y, z = box_coords3(b, bps)
    c = 2 * bps
    offs = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
    return [box_lin3(2 * x + a, 2 * y + bb, 2 * z + cc, c) for a, bb, cc in offs]


def parent_box3(b, ell):                                   # tree3d_common.cpp:120-125
    bps = 1 << ell
    x, y, z = box_coords3(b, bps)
    return box_lin3(x // 2, y // 2, z // 2, bps // 2)


def _face_children_of_box(b, ell, parity):                 # tree3d_common.cpp:73-115
    s = set()
    for c in child_boxes3(b, ell):
        for f in nbor_faces_of_box(c, ell + 1):
            if f == -1:
                continue
            x, y, z = face_coords(f, ell + 1)
            t = face_type(f, ell + 1)
            if (t == XN and x % 2 == parity) or (t == YN and y % 2 == parity) or \
               (t == ZN and z % 2 == parity):
                s.add(f)
    return sorted(s)


# ----------------------------------------------------------------------------
# The factorization (src/DE/mf2d.cpp, src/DE/mf3d.cpp)
# ----------------------------------------------------------------------------
class _Box:
    # A12_asm / A11_asm keep the assembled blocks before elimination (the
    # reference overwrites them); tests compare assembly against them.
    __slots__ = ("int", "bd", "A22", "lu", "XL", "XR", "S", "A11post", "A12_asm", "A11_asm")

    def __init__(self):
        self.int = []
        self.bd = []
        self.A22 = self.lu = self.XL = self.XR = self.S = self.A11post = None
        self.A12_asm = self.A11_asm = None


class _Sep:
    __slots__ = ("dofs", "A11", "A11_base")

    def __init__(self):
        self.dofs = []
        self.A11 = None
        self.A11_base = None     # value before the boxes' Schur complements are added


class MFOracle:
    """Restatement of TreeFactor2D::MF2D / TreeFactor3D::MF3D for Scalar=double.

    A is a scipy.sparse CSR matrix; N = (Nx, Ny) or (Nx, Ny, Nz)."""

    def __init__(self, A, N, width=1, max_side=4, symmetric_schur=False):
        # symmetric_schur: replace every Schur complement by the symmetric
        # matrix built from its lower triangle.  Off by default (the reference
        # keeps the slightly unsymmetric LU result); tests that compare
        # assembly maps against a lower-triangle store turn it on.
        self.symmetric_schur = bool(symmetric_schur)
        self.dim = len(N)
        self.N = tuple(int(n) for n in N)
        self.w = int(width)
        self.A = A.tocsr()
        self._dense_rows = {}
        # tree depth (mf2d.cpp:23-31, mf3d.cpp:41-51)
        top = max(self.N)
        self.levels = int(math.ceil(math.log2((top + width) / (max_side + width))))
        if self.levels <= 1:
            raise RuntimeError("Based on the input parameters, the recursion depth is 1 level")
        L = self.levels
        bps = 1 << (L - 1)
        # leaf widths (mf2d.cpp:57-58)
        self.bw = [int(math.floor((n - (bps - 1) * width) / bps)) for n in self.N]
        for n, b in zip(self.N, self.bw):
            if n < b * (bps - 1) + width * (bps - 1):
                raise RuntimeError("leaf box math broke on this input")
        nbox = lambda ell: (1 << ell) ** self.dim
        self.boxes = [[_Box() for _ in range(nbox(ell))] for ell in range(L)]
        nsep = (lambda b: 2 * b * b - 2 * b) if self.dim == 2 else (lambda b: 3 * b * b * (b - 1))
        # seps[ell] holds separators bounding level-ell boxes (ell >= 1)
        self.seps = [None] + [[_Sep() for _ in range(nsep(1 << ell))] for ell in range(1, L)]
        self.marked_boxes = set()
        self.marked_seps = set()
        self._setup_leaves()

    # -- geometry helpers ---------------------------------------------------
    def _lin(self, i, j, k=0):
        Nx, Ny = self.N[0], self.N[1]
        return i + j * Nx + k * Nx * Ny

    def _bwidth(self, ell, axis, below=False):
        d = self.levels - 1 - ell - (1 if below else 0)
        return self.bw[axis] * (1 << d) + ((1 << d) - 1) * self.w

    def _nbor_seps(self, b, ell):
        return nbor_edges_of_box(b, ell) if self.dim == 2 else nbor_faces_of_box(b, ell)

    def _nbor_boxes(self, e, ell):
        return nbor_boxes_of_edge(e, ell) if self.dim == 2 else nbor_boxes_of_face(e, ell)

    def _child_seps(self, e, ell):
        return child_edges(e, ell) if self.dim == 2 else child_faces(e, ell)

    def _child_boxes(self, b, ell):
        return child_boxes2(b, ell) if self.dim == 2 else child_boxes3(b, ell)

    def _parent(self, b, ell):
        return parent_box2(b, ell) if self.dim == 2 else parent_box3(b, ell)

    def _self_children(self, b, ell):
        return self_edge_children(b, ell) if self.dim == 2 else _face_children_of_box(b, ell, 0)

    def _shared_children(self, b, ell):
        return shared_edge_children(b, ell) if self.dim == 2 else _face_children_of_box(b, ell, 1)

    def _setup_leaves(self):                                # mf2d.cpp:73-133, mf3d.cpp:96-188
        L, w = self.levels, self.w
        ell = L - 1
        bps = 1 << ell
        N, bw = self.N, self.bw
        for b in range(len(self.boxes[ell])):
            self.marked_boxes.add(b)
            if self.dim == 2:
                x, y = box_coords2(b, bps)
                c = (x, y)
            else:
                c = box_coords3(b, bps)
            first = [c[a] * (bw[a] + w) for a in range(self.dim)]
            ub = [N[a] if c[a] == bps - 1 else first[a] + bw[a] for a in range(self.dim)]
            box = self.boxes[ell][b]
            if self.dim == 2:
                box.int = [self._lin(i, j) for j in range(first[1], ub[1]) for i in range(first[0], ub[0])]
            else:
                box.int = [self._lin(i, j, k) for k in range(first[2], ub[2])
                           for j in range(first[1], ub[1]) for i in range(first[0], ub[0])]
            seps = self._nbor_seps(b, ell)
            # each separator is filled once, by the box on its +side:
            # 2D left(0) and top(3); 3D left(0), top(3), below(4)
            fills = [(0, 0), (1, 3)] if self.dim == 2 else [(0, 0), (1, 3), (2, 4)]
            for axis, slot in fills:
                if self.dim == 2:
                    if axis == 0 and c[0] == 0:
                        continue
                    if axis == 1 and c[1] == bps - 1:
                        continue
                else:
                    if axis == 0 and c[0] == 0:
                        continue
                    if axis == 1 and c[1] == bps - 1:
                        continue
                    if axis == 2 and c[2] == 0:
                        continue
                lo = list(first)
                hi = list(ub)
                if axis == 0:
                    lo[0] = first[0] - w
                    hi[0] = lo[0] + w
                elif axis == 1:
                    lo[1] = ub[1]
                    hi[1] = lo[1] + w
                else:
                    lo[2] = first[2] - w
                    hi[2] = lo[2] + w
                dofs = self.seps[ell][seps[slot]].dofs
                if self.dim == 2:
                    dofs.extend(self._lin(i, j) for j in range(lo[1], hi[1]) for i in range(lo[0], hi[0]))
                else:
                    dofs.extend(self._lin(i, j, k) for k in range(lo[2], hi[2])
                                for j in range(lo[1], hi[1]) for i in range(lo[0], hi[0]))

    # -- centre points ------------------------------------------------------
    def _block(self, lo, hi):
        if self.dim == 2:
            return [self._lin(i, j) for j in range(lo[1], hi[1]) for i in range(lo[0], hi[0])]
        return [self._lin(i, j, k) for k in range(lo[2], hi[2])
                for j in range(lo[1], hi[1]) for i in range(lo[0], hi[0])]

    def box_centers(self, b, ell):                          # mf2d.cpp:186-218, mf3d.cpp:253-348
        w, bps = self.w, 1 << ell
        BW = [self._bwidth(ell, a) for a in range(self.dim)]
        BB = [self._bwidth(ell, a, True) for a in range(self.dim)]
        if self.dim == 2:
            x, y = box_coords2(b, bps)
            lo = [x * (BW[0] + w) + BB[0], y * (BW[1] + w) + BB[1]]
            return self._block(lo, [lo[0] + w, lo[1] + w])
        c = box_coords3(b, bps)
        s = set()
        for axis in range(3):               # the line along `axis`
            lo, hi = [], []
            for a in range(3):
                if a == axis:
                    l = c[a] * (BW[a] + w)
                    h = self.N[a] if c[a] == bps - 1 else l + BW[a]
                else:
                    l = c[a] * (BW[a] + w) + BB[a]
                    h = l + w
                lo.append(l)
                hi.append(h)
            s.update(self._block(lo, hi))
        return sorted(s)

    def sep_centers(self, e, ell):                          # mf2d.cpp:220-270, mf3d.cpp:350-524
        w, bps = self.w, 1 << ell
        BW = [self._bwidth(ell, a) for a in range(self.dim)]
        BB = [self._bwidth(ell, a, True) for a in range(self.dim)]
        if self.dim == 2:
            x, y = edge_coords(e, ell)
            if edge_type(e, ell) == L2R:
                lo = [x * (BW[0] + w) + BB[0], y * (BW[1] + w) + BW[1]]
            else:
                lo = [x * (BW[0] + w) + BW[0], y * (BW[1] + w) + BB[1]]
            return self._block(lo, [lo[0] + w, lo[1] + w])
        c = face_coords(e, ell)
        t = face_type(e, ell)
        normal = {XN: 0, YN: 1, ZN: 2}[t]
        s = set()
        for axis in range(3):
            if axis == normal:
                continue
            lo, hi = [], []
            for a in range(3):
                if a == normal:
                    l = c[a] * (BW[a] + w) + BW[a]
                    h = l + w
                elif a == axis:
                    l = c[a] * (BW[a] + w)
                    h = self.N[a] if c[a] == bps - 1 else l + BW[a]
                else:
                    l = c[a] * (BW[a] + w) + BB[a]
                    h = l + w
                lo.append(l)
                hi.append(h)
            s.update(self._block(lo, hi))
        return sorted(s)

    # -- sparse helpers -----------------------------------------------------
    def _sub(self, rows, cols):                             # sparse.cpp:95-116
        if len(rows) == 0 or len(cols) == 0:
            return np.zeros((len(rows), len(cols)))
        return self.A[np.asarray(rows)][:, np.asarray(cols)].toarray()

    @staticmethod
    def _table(big, small):
        pos = {d: i for i, d in enumerate(big)}
        t1, t2 = [], []
        for i, d in enumerate(small):
            p = pos.get(d)
            if p is not None:
                t1.append(p)
                t2.append(i)
        return np.asarray(t1, np.int64), np.asarray(t2, np.int64)

    def _scatter_add(self, A, big, B, small):               # mf2d.cpp:755-776
        t1, t2 = self._table(big, small)
        A[np.ix_(t1, t1)] += B[np.ix_(t2, t2)]

    def _scatter_replace(self, A, big, B, small):           # mf2d.cpp:778-800
        t1, t2 = self._table(big, small)
        A[np.ix_(t1, t1)] = B[np.ix_(t2, t2)]

    def _scatter_replace2(self, A, rowbig, colbig, B, small):  # mf2d.cpp:804-834
        r1, r2 = self._table(rowbig, small)
        c1, c2 = self._table(colbig, small)
        A[np.ix_(r1, c1)] = B[np.ix_(r2, c2)]

    def _add_new(self, A, total, new):                      # mf2d.cpp:836-862
        pos = {d: i for i, d in enumerate(total)}
        table = np.asarray([pos[d] for d in new], np.int64)
        flags = np.zeros(len(total), bool)
        flags[table] = True
        A[:, table] += self._sub(total, new)
        other = np.nonzero(~flags)[0]
        # A(table[j], i) += A_(new[j], total[i]) for i not a new DOF (i != table[j] holds)
        A[np.ix_(table, other)] += self._sub(new, [total[i] for i in other])

    def _add_new_rows(self, A, rows, cols, new):            # mf2d.cpp:864-882
        pos = {d: i for i, d in enumerate(rows)}
        table = np.asarray([pos[d] for d in new], np.int64)
        A[table, :] += self._sub(new, cols)

    def _add_new_cols(self, A, rows, cols, new):            # mf2d.cpp:884-901
        pos = {d: i for i, d in enumerate(cols)}
        table = np.asarray([pos[d] for d in new], np.int64)
        A[:, table] += self._sub(rows, new)

    # -- dense kernels (dense.hpp:180-227) ------------------------------------
    def _eliminate(self, A22, A12, A21):
        lu = sla.lu_factor(A22, check_finite=False)
        XL = sla.lu_solve(lu, A12.T, trans=1, check_finite=False).T   # X A22 = A12
        XR = sla.lu_solve(lu, A21, check_finite=False)
        S = -(A12 @ XR)
        if self.symmetric_schur:
            S = np.tril(S) + np.tril(S, -1).T
        return lu, XL, XR, S

    # -- levels ---------------------------------------------------------------
    def factor(self):                                       # mf2d.cpp:449-500
        self._factor_leaf()
        for ell in range(self.levels - 2, -1, -1):
            if ell != 0:
                self._update_seps(ell)
            self._update_boxes(ell)
            self._factor_upper(ell)

    def _factor_leaf(self):                                 # mf2d.cpp:504-626
        ell = self.levels - 1
        for b in sorted(self.marked_boxes):
            box = self.boxes[ell][b]
            seps = self._nbor_seps(b, ell)
            box.bd = []
            for e in seps:
                if e != -1:
                    box.bd.extend(self.seps[ell][e].dofs)
            box.A22 = self._sub(box.int, box.int)
            A21 = self._sub(box.int, box.bd)
            A12 = self._sub(box.bd, box.int)
            box.lu, box.XL, box.XR, box.S = self._eliminate(box.A22, A12, A21)
            box.A11post = self._sub(box.bd, box.bd) + box.S
            self.marked_seps.update(seps)
        self.marked_boxes = set()
        self._accumulate_seps(ell, leaf=True)

    def _accumulate_seps(self, ell, leaf):                  # mf2d.cpp:582-620, 708-747
        new_marked = set()
        for e in sorted(self.marked_seps):
            if e == -1:
                continue
            sep = self.seps[ell][e]
            if leaf:
                sep.A11 = self._sub(sep.dofs, sep.dofs)
                sep.A11_base = sep.A11.copy()
            for b in self._nbor_boxes(e, ell):
                box = self.boxes[ell][b]
                self._scatter_add(sep.A11, sep.dofs, box.S, box.bd)
                p = self._parent(b, ell)
                self.marked_boxes.add(p)
                if ell > 1:
                    new_marked.update(self._nbor_seps(p, ell - 1))
        self.marked_seps = new_marked

    def _update_seps(self, ell):                            # mf2d.cpp:274-319
        for e in sorted(self.marked_seps):
            if e == -1:
                continue
            sep = self.seps[ell][e]
            kids = self._child_seps(e, ell)
            sep.dofs = []
            for c in kids:
                sep.dofs.extend(self.seps[ell + 1][c].dofs)
            centers = self.sep_centers(e, ell)
            sep.dofs.extend(centers)
            sep.A11 = np.zeros((len(sep.dofs), len(sep.dofs)))
            self._add_new(sep.A11, sep.dofs, centers)
            for c in kids:
                ch = self.seps[ell + 1][c]
                self._scatter_replace(sep.A11, sep.dofs, ch.A11, ch.dofs)
            sep.A11_base = sep.A11.copy()
        self.marked_seps = set()

    def _update_boxes(self, ell):                           # mf2d.cpp:322-446
        for b in sorted(self.marked_boxes):
            box = self.boxes[ell][b]
            self_kids = self._self_children(b, ell)
            box.int = []
            for c in self_kids:
                box.int.extend(self.seps[ell + 1][c].dofs)
            centers = self.box_centers(b, ell)
            box.int.extend(centers)
            n = len(box.int)
            A22 = np.zeros((n, n))
            self._add_new(A22, box.int, centers)
            nb = self._nbor_seps(b, ell)
            box.bd = []
            for e in nb:
                if e != -1:
                    box.bd.extend(self.seps[ell][e].dofs)
            m = len(box.bd)
            A11 = np.zeros((m, m))
            A12 = np.zeros((m, n))
            A21 = np.zeros((n, m))
            for e in nb:
                if e == -1:
                    continue
                cp = self.sep_centers(e, ell)
                self._add_new_rows(A12, box.bd, box.int, cp)
                self._add_new_cols(A21, box.int, box.bd, cp)
            for c in self._child_boxes(b, ell):
                ch = self.boxes[ell + 1][c]
                self._scatter_replace2(A12, box.bd, box.int, ch.A11post, ch.bd)
                self._scatter_replace2(A21, box.int, box.bd, ch.A11post, ch.bd)
                self._scatter_replace(A22, box.int, ch.A11post, ch.bd)
                self._scatter_replace(A11, box.bd, ch.A11post, ch.bd)
            for c in self_kids:
                ch = self.seps[ell + 1][c]
                self._scatter_replace(A22, box.int, ch.A11, ch.dofs)
            for c in self._shared_children(b, ell):
                ch = self.seps[ell + 1][c]
                self._scatter_replace(A11, box.bd, ch.A11, ch.dofs)
            box.A22 = A22
            box.A11post = A11
            box.A12_asm = A12.copy()
            box.A11_asm = A11.copy()
            box.XL = A12     # the reference parks A12/A21 in XL/XR until factoring
            box.XR = A21

    def _factor_upper(self, ell):                           # mf2d.cpp:628-753
        if ell == 0:
            root = self.boxes[0][0]
            root.lu = sla.lu_factor(root.A22, check_finite=False)
            return
        for b in sorted(self.marked_boxes):
            box = self.boxes[ell][b]
            A12, A21 = box.XL, box.XR
            box.lu, box.XL, box.XR, box.S = self._eliminate(box.A22, A12, A21)
            box.A11post = box.A11post + box.S
            self.marked_seps.update(self._nbor_seps(b, ell))
        self.marked_boxes = set()
        self._accumulate_seps(ell, leaf=False)

    # -- localized update (mf2d.cpp:150-181, mf3d.cpp:208-248) ---------------
    def update(self, A, modified):
        self.marked_boxes = set()
        self.marked_seps = set()
        self.A = A.tocsr()
        ell = self.levels - 1
        bps = 1 << ell
        Nx, Ny = self.N[0], self.N[1]
        for idx in sorted(set(int(d) for d in modified)):
            i = idx % Nx
            r = idx // Nx
            crd = [i, r] if self.dim == 2 else [i, r % Ny, r // Ny]
            # i / (b + w) as in the reference; clamped to the last box, which
            # absorbs the remainder when (b + w) does not divide N (there the
            # reference's quotient can reach bps and name the wrong box).
            bc = [min(crd[a] // (self.bw[a] + self.w), bps - 1) for a in range(self.dim)]
            if self.dim == 2:
                self.marked_boxes.add(bc[0] + bc[1] * bps)
            else:
                self.marked_boxes.add(box_lin3(bc[0], bc[1], bc[2], bps))
        self.factor()

    # -- solve / apply (mf2d.cpp:904-1054) -------------------------------------
    def solve(self, b):
        b = np.array(b, np.float64, copy=True)
        L = self.levels
        for ell in range(L - 1, 0, -1):
            for box in self.boxes[ell]:
                rd, sk = np.asarray(box.int), np.asarray(box.bd)
                b_rd = b[rd]
                if len(sk):
                    b[sk] = b[sk] - box.XL @ b_rd
                b[rd] = sla.lu_solve(box.lu, b_rd, check_finite=False)
        root = self.boxes[0][0]
        rd = np.asarray(root.int)
        b[rd] = sla.lu_solve(root.lu, b[rd], check_finite=False)
        for ell in range(1, L):
            for box in self.boxes[ell]:
                rd, sk = np.asarray(box.int), np.asarray(box.bd)
                if len(sk):
                    b[rd] = b[rd] - box.XR @ b[sk]
        return b

    def apply(self, x):
        b = np.array(x, np.float64, copy=True)
        L = self.levels
        for ell in range(L - 1, 0, -1):
            for box in self.boxes[ell]:
                rd, sk = np.asarray(box.int), np.asarray(box.bd)
                b_rd = b[rd]
                if len(sk):
                    b_rd = b_rd + box.XR @ b[sk]
                b[rd] = box.A22 @ b_rd
        root = self.boxes[0][0]
        rd = np.asarray(root.int)
        b[rd] = root.A22 @ b[rd]
        for ell in range(1, L):
            for box in self.boxes[ell]:
                rd, sk = np.asarray(box.int), np.asarray(box.bd)
                if len(sk):
                    b[sk] = b[sk] + box.XL @ b[rd]
        return b


def box_lin_any(x, y, z, bps, dim):
    return x + y * bps if dim == 2 else box_lin3(x, y, z, bps)


def front_sizes(oracle):
    """[(level, box, n, m)] of a factored oracle."""
    out = []
    for ell, boxes in enumerate(oracle.boxes):
        for b, box in enumerate(boxes):
            out.append((ell, b, len(box.int), len(box.bd)))
    return out
