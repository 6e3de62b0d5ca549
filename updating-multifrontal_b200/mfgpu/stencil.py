"""Variable-coefficient 5-point (2D) / 7-point (3D) Laplacian in CSR form, and the
seeded coefficient fields and right-hand sides the workloads use.

`build_laplacian` follows the reference fixture
(test_include/DE/buildLaplacian.hpp:10-132 for 2D, :244-391 for 3D): the
coefficient array is node-valued with shape (Nx+2w, Ny+2w[, Nz+2w]) indexed
[i][j][k] like the reference's nested vectors; a face coefficient is the
arithmetic mean of its two nodes; the off-diagonal is coef*ahalf/h^2 and the
diagonal minus the sum of the same face terms.  Every value is produced by the
same sequence of IEEE double operations as the reference loop, so the CSR is
bit-identical, and entries within a row are in ascending column order.
"""
import numpy as np

# Stencil coefficient tables for widths 1..3 (buildLaplacian.hpp:20-35).
_COEFFS = {
    1: [0.0, -1.0],
    2: [0.0, -4.0 / 3.0, 1.0 / 12.0],
    3: [0.0, -3.0 / 2.0, 3.0 / 20.0, -1.0 / 90.0],
}


class CSR:
    """Plain CSR container (row_ptr int32, col_ind int32, val float64)."""

    def __init__(self, row_ptr, col_ind, val, n):
        self.row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        self.col_ind = np.ascontiguousarray(col_ind, np.int32)
        self.val = np.ascontiguousarray(val, np.float64)
        self.n = int(n)

    @property
    def nnz(self):
        return int(self.row_ptr[-1])

    def matvec(self, x):
        """y = A x in float64 (numpy; row sums in CSR order)."""
        x = np.asarray(x, np.float64)
        prod = self.val * x[self.col_ind]
        return np.add.reduceat(prod, self.row_ptr[:-1]) if self.n else prod[:0]

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col_ind, self.row_ptr), shape=(self.n, self.n))


def _axis_terms(a, W, axis, k, sl_self):
    """ahalf values towards -k and +k along `axis` for every grid node."""
    dim = a.ndim

    def take(off):
        idx = []
        for d in range(dim):
            s = sl_self[d]
            if d == axis:
                idx.append(slice(s.start + off, s.stop + off))
            else:
                idx.append(s)
        return a[tuple(idx)]

    minus = 0.5 * (take(-k) + take(-k + 1))   # 0.5*(A[..-k] + A[..-k+1])
    plus = 0.5 * (take(k) + take(k - 1))      # 0.5*(A[..+k] + A[..+k-1])
    return minus, plus


def build_laplacian(a, width=1, h=None):
    """CSR of -div(a grad u) on an Nx x Ny (x Nz) grid, DOF id i + j*Nx (+ k*Nx*Ny).

    `a` has shape (Nx+2w, Ny+2w) or (Nx+2w, Ny+2w, Nz+2w)."""
    a = np.asarray(a, np.float64)
    dim = a.ndim
    W = int(width)
    if W not in _COEFFS:
        raise ValueError("width must be 1, 2 or 3")
    c = _COEFFS[W]
    N = [s - 2 * W for s in a.shape]
    if h is None:
        h = (1.0,) * dim
    hh = [float(x) * float(x) for x in h]
    sl_self = [slice(W, W + N[d]) for d in range(dim)]
    # per-axis, per-k face terms on the (Nx, Ny[, Nz]) node grid (x-major arrays)
    terms = {}
    for axis in range(dim):
        for k in range(1, W + 1):
            terms[(axis, k)] = _axis_terms(a, W, axis, k, sl_self)

    # diagonal: v = 0; for k = W..1: v -= c*(ah1+ah2)/hhx; v -= c*(ah3+ah4)/hhy; ...
    diag = np.zeros(N, np.float64)
    for k in range(W, 0, -1):
        for axis in range(dim):
            mi, pl = terms[(axis, k)]
            diag = diag - (c[k] * (mi + pl)) / hh[axis]

    # Column entries of each row, in the reference's push order, which is also
    # ascending column order: for 3D back(z), down(y), left(x), self, right(x),
    # up(y), front(z); 2D drops z.
    order_minus = list(range(dim - 1, -1, -1))       # z, y, x  /  y, x
    order_plus = list(range(dim))                    # x, y, z
    strides = [1, N[0], N[0] * (N[1] if dim > 1 else 1)]
    grids = np.meshgrid(*[np.arange(n) for n in N], indexing="ij")
    lin = grids[0].astype(np.int64)
    for d in range(1, dim):
        lin = lin + grids[d].astype(np.int64) * strides[d]
    cols, vals, oks = [], [], []
    for axis in order_minus:
        for k in range(W, 0, -1):
            mi, _ = terms[(axis, k)]
            cols.append(lin - k * strides[axis])
            vals.append((c[k] * mi) / hh[axis])
            oks.append(grids[axis] - k >= 0)
    cols.append(lin)
    vals.append(diag)
    oks.append(np.ones(N, bool))
    for axis in order_plus:
        for k in range(1, W + 1):
            _, pl = terms[(axis, k)]
            cols.append(lin + k * strides[axis])
            vals.append((c[k] * pl) / hh[axis])
            oks.append(grids[axis] + k <= N[axis] - 1)

    # Flatten in DOF order: DOF id is x-fastest, so transpose grids to (z, y, x).
    def flat(arr):
        return np.ascontiguousarray(np.transpose(arr)).reshape(-1)

    C = np.stack([flat(x) for x in cols], axis=1)
    V = np.stack([flat(x) for x in vals], axis=1)
    M = np.stack([flat(x) for x in oks], axis=1)
    counts = M.sum(axis=1)
    row_ptr = np.zeros(C.shape[0] + 1, np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    return CSR(row_ptr.astype(np.int32), C[M].astype(np.int32), V[M], C.shape[0])


def coef_shape(N, width=1):
    return tuple(int(n) + 2 * width for n in N)


def uniform_coefficients(N, width=1, value=1.0):
    return np.full(coef_shape(N, width), float(value))


def loguniform_coefficients(N, lo, hi, seed, width=1):
    """Node coefficients a = lo * (hi/lo)**U, U ~ U[0,1) from numpy PCG64(seed)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    u = rng.random(coef_shape(N, width))
    return lo * np.power(hi / lo, u)


def uniform_rhs(n, nrhs, seed):
    """nrhs right-hand sides, iid uniform[-1, 1), shape (nrhs, n)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.uniform(-1.0, 1.0, size=(nrhs, n))


def scale_box(a, lo_corner, side, factor, width=1):
    """Copy of `a` with cells [lo, lo+side) (grid coordinates) multiplied by factor.

    Cell (i, j[, k]) of the grid is node (i+w, j+w[, k+w]) of the coefficient array."""
    b = np.array(a, copy=True)
    idx = tuple(slice(int(l) + width, int(l) + width + int(s))
                for l, s in zip(lo_corner, side if np.ndim(side) else [side] * a.ndim))
    b[idx] = b[idx] * factor
    return b


def modified_dofs(A1, A2):
    """Columns of entries whose values differ, as test_src/DE/testMF2D.cpp:143-150."""
    if A1.nnz != A2.nnz or not np.array_equal(A1.col_ind, A2.col_ind):
        raise ValueError("sparsity patterns differ")
    diff = A1.val != A2.val
    return np.unique(A1.col_ind[diff]).astype(np.int32)
