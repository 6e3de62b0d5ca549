"""B200 multifrontal factor / localized update / solve (Python binding).

`MF2D` / `MF3D` mirror the reference's TreeFactor2D::MF2D<double> and
TreeFactor3D::MF3D<double> (include/DE/mf.hpp:67-80, 173-188): a constructor
taking the CSR matrix, grid sizes, separator width and leaf parameter, then
Factor(), Update(A, modifiedDOFs), Solve(b) and Apply(x).  Errors follow the
reference: a too-shallow tree or broken leaf arithmetic raise RuntimeError
(the reference throws std::runtime_error, src/DE/mf2d.cpp:42,64); a matrix
that is not symmetric positive definite raises RuntimeError from Factor();
bad arguments raise ValueError.  All compute runs in libmfgpu.so on the GPU;
there is no CPU path.
"""
import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import MFGPU_FP64, MFGPU_MIXED, TASK_DTYPE
from .stencil import CSR, build_laplacian

__all__ = ["MF2D", "MF3D", "MFBatch", "Server", "Symbolic", "CSR", "build_laplacian", "MFGPU_FP64",
           "MFGPU_MIXED", "MFError", "inject_alloc_failure"]


def _as_csr(A):
    """A as this package's CSR: a CSR (of this or another copy of the stencil
    module: anything with row_ptr / col_ind / val / n) or a scipy sparse matrix."""
    if isinstance(A, CSR):
        return A
    if all(hasattr(A, k) for k in ("row_ptr", "col_ind", "val", "n")):
        return CSR(A.row_ptr, A.col_ind, A.val, A.n)
    A = A.tocsr()
    return CSR(A.indptr, A.indices, A.data, A.shape[0])


def inject_alloc_failure(after):
    """Test hook: the next `after` device allocations succeed, the one after
    fails as out of memory (MFGPU_ERR_OOM); after < 0 disarms."""
    _lib.load().mfgpu_inject_alloc_failure(int(after))


class MFError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{_lib.status_string(status)}: {msg}")
        self.status = status


def _raise(status, msg):
    if status in (_lib.MFGPU_ERR_DEPTH, _lib.MFGPU_ERR_LEAF):
        raise RuntimeError(msg)
    if status == _lib.MFGPU_ERR_ARG:
        raise ValueError(msg)
    raise MFError(status, msg)


class _MFBase:
    _dim = None

    def __init__(self, A, N, width=1, max_side_length=4, precision=MFGPU_FP64, device=0,
                 refine_tol=1e-10, refine_maxit=50):
        lib = _lib.load()
        A = _as_csr(A)
        self.A = A
        self.N = tuple(int(x) for x in N)
        opts = _lib.default_options(precision, device, refine_tol, refine_maxit)
        h = C.c_void_p()
        Nz = self.N[2] if self._dim == 3 else 1
        st = lib.mfgpu_create(self._dim, self.N[0], self.N[1], Nz, int(width), int(max_side_length),
                              int(A.n), _lib._ptr(A.row_ptr), _lib._ptr(A.col_ind), _lib._ptr(A.val),
                              C.byref(opts), C.byref(h))
        if st != _lib.MFGPU_OK:
            _raise(st, lib.mfgpu_last_error(None).decode())
        self._h = h
        self._lib = lib

    def _check(self, st):
        if st != _lib.MFGPU_OK:
            _raise(st, self._lib.mfgpu_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mfgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the reference's public members ------------------------------------
    def Factor(self):
        self._check(self._lib.mfgpu_factor(self._h))

    def Update(self, A, modifiedDOFs):
        A = _as_csr(A)
        mod = np.ascontiguousarray(sorted(set(int(d) for d in modifiedDOFs)), np.int32)
        self._check(self._lib.mfgpu_update(self._h, _lib._ptr(A.val), A.nnz, _lib._ptr(mod),
                                           len(mod)))
        self.A = A

    def _vec_op(self, v, fn):
        v = np.asarray(v, np.float64)
        one = v.ndim == 1
        X = np.asfortranarray(v.reshape(-1, 1) if one else v)
        if X.shape[0] != self.A.n:
            raise ValueError("vector length does not match the matrix")
        out = np.empty_like(X, order="F")
        self._check(fn(self._h, X.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p),
                       X.shape[1], X.shape[0]))
        return out[:, 0] if one else out

    def Solve(self, b):
        """x = A^{-1} b for b of shape (n,) or (n, nrhs)."""
        return self._vec_op(b, self._lib.mfgpu_solve)

    def Apply(self, x):
        """b = (factored A) x for x of shape (n,) or (n, nrhs)."""
        return self._vec_op(x, self._lib.mfgpu_apply)

    # -- extras ----------------------------------------------------------
    def refactor(self, val):
        """Replace every matrix value (same pattern) and refactor all fronts."""
        val = np.ascontiguousarray(val, np.float64)
        self._check(self._lib.mfgpu_refactor(self._h, _lib._ptr(val), val.size))

    def refactor_device(self, val_ptr, nnz):
        self._check(self._lib.mfgpu_refactor_device(self._h, C.c_void_p(val_ptr), nnz))

    def update_device(self, val_ptr, nnz, modifiedDOFs):
        mod = np.ascontiguousarray(sorted(set(int(d) for d in modifiedDOFs)), np.int32)
        self._check(self._lib.mfgpu_update_device(self._h, C.c_void_p(val_ptr), nnz,
                                                  _lib._ptr(mod), len(mod)))

    def update_host_ptr(self, val_ptr, nnz, mod):
        """Update from a raw host pointer (e.g. pinned memory); mod int32 array."""
        self._check(self._lib.mfgpu_update(self._h, C.c_void_p(val_ptr), nnz, _lib._ptr(mod),
                                           len(mod)))

    def refactor_host_ptr(self, val_ptr, nnz):
        self._check(self._lib.mfgpu_refactor(self._h, C.c_void_p(val_ptr), nnz))

    def solve_host_ptr(self, b_ptr, x_ptr, nrhs, ld):
        self._check(self._lib.mfgpu_solve(self._h, C.c_void_p(b_ptr), C.c_void_p(x_ptr), nrhs, ld))

    def profile(self, on=True):
        self._check(self._lib.mfgpu_profile_enable(self._h, 1 if on else 0))

    def profile_reset(self):
        self._check(self._lib.mfgpu_profile_reset(self._h))

    def profile_read(self):
        out = {}
        for i, nm in enumerate(_lib.KERNEL_CLASSES):
            la, ms, fl, by = C.c_int64(), C.c_double(), C.c_double(), C.c_double()
            self._check(self._lib.mfgpu_profile_read(self._h, i, C.byref(la), C.byref(ms),
                                                     C.byref(fl), C.byref(by)))
            out[nm] = dict(launches=la.value, ms=ms.value, flops=fl.value, bytes=by.value)
        return out

    @staticmethod
    def kernel_launches():
        return int(_lib.load().mfgpu_kernel_launches())

    def solve_device(self, b_ptr, x_ptr, nrhs, ld):
        self._check(self._lib.mfgpu_solve_device(self._h, C.c_void_p(b_ptr), C.c_void_p(x_ptr),
                                                 nrhs, ld))

    def apply_device(self, x_ptr, b_ptr, nrhs, ld):
        self._check(self._lib.mfgpu_apply_device(self._h, C.c_void_p(x_ptr), C.c_void_p(b_ptr),
                                                 nrhs, ld))

    def stencil_assemble_device(self, coef_ptr, val_ptr, h=(1.0, 1.0, 1.0)):
        """CSR values of the handle's stencil from device coefficients (bit-exact
        with stencil.build_laplacian) into the device array at val_ptr."""
        hh = np.ascontiguousarray(h, np.float64)
        self._check(self._lib.mfgpu_stencil_assemble_device(self._h, C.c_void_p(coef_ptr),
                                                            _lib._ptr(hh), C.c_void_p(val_ptr)))

    def stencil_update_device(self, coef_ptr, lo, hi, val_ptr, h=(1.0, 1.0, 1.0)):
        """Recompute the rows touched by the cell box [lo, hi) in place; returns
        the modified DOFs (sorted int32 array)."""
        hh = np.ascontiguousarray(h, np.float64)
        lo3 = np.ascontiguousarray(list(lo) + [0] * (3 - len(lo)), np.int32)
        hi3 = np.ascontiguousarray(list(hi) + [1] * (3 - len(hi)), np.int32)
        # at most every row of the box grown by one cell changes; one call
        # (the values are updated in place, so a second call would find nothing)
        cap = 1
        for d in range(len(lo)):
            cap *= max(0, int(hi[d]) + 1 - max(int(lo[d]) - 1, 0))
        cap = max(1, min(cap, self.A.n))
        out = np.zeros(cap, np.int32)
        cnt = C.c_int()
        self._check(self._lib.mfgpu_stencil_update_device(
            self._h, C.c_void_p(coef_ptr), _lib._ptr(hh), _lib._ptr(lo3), _lib._ptr(hi3),
            C.c_void_p(val_ptr), _lib._ptr(out), len(out), C.byref(cnt)))
        return out[:cnt.value]

    def save(self, path):
        """Write the factorization to a file (mfgpu_save); load() restores it
        into a handle built for the same problem, with no Factor() needed."""
        self._check(self._lib.mfgpu_save(self._h, os.fsencode(path)))

    def load(self, path):
        """Restore a factorization written by save() (mfgpu_load)."""
        self._check(self._lib.mfgpu_load(self._h, os.fsencode(path)))

    LEVEL_KERNELS = {-1: "none", 0: "fused", 1: "coop", 2: "tc", 3: "stepped", 4: "lu", 5: "panel"}

    def autotune(self, reps=2):
        """Full factorization that times each level's eligible kernels and keeps
        the fastest for later full factorizations (mfgpu_autotune).  Returns
        the kernel chosen per level, root first."""
        out = np.zeros(self.info()["levels"], np.int32)
        self._check(self._lib.mfgpu_autotune(self._h, int(reps), _lib._ptr(out)))
        return [self.LEVEL_KERNELS[int(k)] for k in out]

    def set_stream(self, stream_ptr):
        self._check(self._lib.mfgpu_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def graphs(self):
        """(factorization graph captured, number of sweep graphs held)."""
        fg, sg = C.c_int(), C.c_int()
        self._check(self._lib.mfgpu_graphs(self._h, C.byref(fg), C.byref(sg)))
        return bool(fg.value), sg.value

    def set_wait_limit(self, polls):
        """Poll limit of the bounded device waits of later calls (0: built-in);
        a wait that gives up raises MFError with status MFGPU_ERR_TIMEOUT."""
        self._check(self._lib.mfgpu_set_wait_limit(self._h, int(polls)))

    def info(self):
        inf = _lib.Info()
        self._check(self._lib.mfgpu_get_info(self._h, C.byref(inf)))
        return {f: (list(getattr(inf, f)) if f == "leaf_box" else getattr(inf, f))
                for f, _ in _lib.Info._fields_}

    def stats(self):
        s = _lib.Stats()
        self._check(self._lib.mfgpu_last_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in _lib.Stats._fields_}


class MFBatch(_MFBase):
    """Independent problems factored and solved together (mfgpu_batch_create).

    `problems` is a list of (A, N, width, maxSideLength) with N = (Nx, Ny) or
    (Nx, Ny, Nz).  The handle works on the block-diagonal matrix: vectors are
    the problems' vectors stacked (row offsets in `self.offsets`); `join` and
    `split` convert.  Update(A_list, mods) takes the new matrices (None keeps a
    problem unchanged) and the per-problem modified DOFs (local numbering).
    """

    def __init__(self, problems, precision=MFGPU_FP64, device=0, refine_tol=1e-10,
                 refine_maxit=50):
        lib = _lib.load()
        mats, geo = [], []
        for A, N, width, ms in problems:
            A = _as_csr(A)
            N = tuple(int(x) for x in N)
            mats.append(A)
            geo.append((len(N), N[0], N[1], N[2] if len(N) == 3 else 1, int(width), int(ms)))
        self.mats = mats
        self.A = _block_diag(mats)
        cols = [np.ascontiguousarray([g[k] for g in geo], np.int32) for k in range(6)]
        opts = _lib.default_options(precision, device, refine_tol, refine_maxit)
        h = C.c_void_p()
        st = lib.mfgpu_batch_create(len(problems), *[_lib._ptr(c) for c in cols], int(self.A.n),
                                    _lib._ptr(self.A.row_ptr), _lib._ptr(self.A.col_ind),
                                    _lib._ptr(self.A.val), C.byref(opts), C.byref(h))
        if st != _lib.MFGPU_OK:
            _raise(st, lib.mfgpu_last_error(None).decode())
        self._h = h
        self._lib = lib
        cnt = C.c_int()
        offs = np.zeros(len(problems) + 1, np.int64)
        self._check(lib.mfgpu_batch_info(h, C.byref(cnt),
                                         offs.ctypes.data_as(C.POINTER(C.c_int64))))
        self.offsets = offs
        self.N = None

    def join(self, vecs, nrhs=None):
        """Stack per-problem right-hand sides ((n_p,) or (n_p, k_p)) into (n, nrhs),
        zero-padding problems with fewer columns."""
        vs = [np.asarray(v, np.float64).reshape(len(v), -1) for v in vecs]
        k = nrhs or max(v.shape[1] for v in vs)
        out = np.zeros((int(self.offsets[-1]), k), order="F")
        for p, v in enumerate(vs):
            out[self.offsets[p]:self.offsets[p + 1], :v.shape[1]] = v
        return out

    def split(self, X):
        return [X[self.offsets[p]:self.offsets[p + 1]] for p in range(len(self.offsets) - 1)]

    def Update(self, A_list, mods):
        """A_list[p]: new matrix of problem p (same pattern) or None; mods[p]: its
        modified DOFs (local numbering)."""
        mats = [self.mats[p] if A is None else _as_csr(A) for p, A in enumerate(A_list)]
        allmod = []
        for p, m in enumerate(mods):
            allmod.extend(int(d) + int(self.offsets[p]) for d in (m if m is not None else ()))
        B = _block_diag(mats)
        mod = np.ascontiguousarray(sorted(set(allmod)), np.int32)
        self._check(self._lib.mfgpu_update(self._h, _lib._ptr(B.val), B.nnz, _lib._ptr(mod),
                                           len(mod)))
        self.mats, self.A = mats, B


class Server:
    """Update-serving loop over a factored MF2D/MF3D (mfgpu_server_create).

    submit(lo, hi, factor, b) queues a request (coefficients of the cell box
    [lo, hi) times `factor`, right-hand sides b of shape (n,) or (n, k)) and
    returns a ticket; wait(ticket) returns (x, info).  Requests are independent:
    each answer is that of the base matrix under its own change.  Queued
    requests are served in batches of at most `slots` whose private root-path
    copies fit in the pool together; a batch's root paths are refactored by
    one set of level launches (info["batch"]: the batch size).
    """

    def __init__(self, F, coef, slots=4, pool_gb=8.0, h=(1.0, 1.0, 1.0)):
        import torch
        self.F = F
        self._lib = F._lib
        self._coef = torch.from_numpy(np.ascontiguousarray(coef, np.float64)).cuda()
        hh = np.ascontiguousarray(h, np.float64)
        srv = C.c_void_p()
        st = self._lib.mfgpu_server_create(F._h, C.c_void_p(self._coef.data_ptr()), _lib._ptr(hh),
                                           int(slots), int(pool_gb * 2 ** 30), C.byref(srv))
        if st != _lib.MFGPU_OK:
            _raise(st, self._lib.mfgpu_last_error(F._h).decode())
        self._srv = srv
        self._pending = {}

    def submit(self, lo, hi, factor, b):
        b = np.asarray(b, np.float64)
        one = b.ndim == 1
        B = np.asfortranarray(b.reshape(-1, 1) if one else b)
        X = np.zeros_like(B, order="F")
        lo3 = np.ascontiguousarray(list(lo) + [0] * (3 - len(lo)), np.int32)
        hi3 = np.ascontiguousarray(list(hi) + [1] * (3 - len(hi)), np.int32)
        t = C.c_int64()
        st = self._lib.mfgpu_server_submit(self._srv, _lib._ptr(lo3), _lib._ptr(hi3), float(factor),
                                           B.ctypes.data_as(C.c_void_p), B.shape[1], B.shape[0],
                                           X.ctypes.data_as(C.c_void_p), C.byref(t))
        if st != _lib.MFGPU_OK:
            _raise(st, "bad request")
        self._pending[t.value] = (B, X, one)     # keep the buffers alive
        return t.value

    def wait(self, ticket):
        info = _lib.RequestInfo()
        st = self._lib.mfgpu_server_wait(self._srv, int(ticket), C.byref(info))
        B, X, one = self._pending.pop(ticket)
        if st != _lib.MFGPU_OK:
            _raise(st, self._lib.mfgpu_server_last_error(self._srv).decode())
        d = {f: getattr(info, f) for f, _ in _lib.RequestInfo._fields_ if f not in ("pad", "reserved")}
        return (X[:, 0] if one else X), d

    def close(self):
        if getattr(self, "_srv", None):
            self._lib.mfgpu_server_destroy(self._srv)
            self._srv = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _block_diag(mats):
    rp, ci, va = [np.zeros(1, np.int32)], [], []
    rows = nnz = 0
    for A in mats:
        rp.append((A.row_ptr[1:].astype(np.int64) + nnz).astype(np.int32))
        ci.append((A.col_ind.astype(np.int64) + rows).astype(np.int32))
        va.append(A.val)
        rows += A.n
        nnz += A.nnz
    return CSR(np.concatenate(rp), np.concatenate(ci), np.concatenate(va), rows)


class MF2D(_MFBase):
    """MF2D(A, Nx, Ny, width=1, maxSideLength=4)."""
    _dim = 2

    def __init__(self, A, Nx, Ny, width=1, maxSideLength=4, **kw):
        super().__init__(A, (Nx, Ny), width, maxSideLength, **kw)


class MF3D(_MFBase):
    """MF3D(A, Nx, Ny, Nz, width=1, maxSideLength=4)."""
    _dim = 3

    def __init__(self, A, Nx, Ny, Nz, width=1, maxSideLength=4, **kw):
        super().__init__(A, (Nx, Ny, Nz), width, maxSideLength, **kw)


class Symbolic:
    """Host-only view of the schedule: DOF lists and assembly tasks."""

    def __init__(self, dim, N, width=1, max_side_length=4, batch=None, full=False):
        """One problem, or with batch=[(dim, N, width, maxSideLength), ...] the
        forest schedule of a batch (dim, N, width, max_side_length ignored).
        full=True: task tables for nonsymmetric matrices (both triangles of
        every block; mfgpu_symbolic_create_full)."""
        lib = _lib.load()
        h = C.c_void_p()
        if batch is not None:
            cols = [np.ascontiguousarray(c, np.int32) for c in zip(
                *[(d, n[0], n[1], n[2] if d == 3 else 1, w, m) for d, n, w, m in batch])]
            st = lib.mfgpu_symbolic_batch_create(len(batch), *[_lib._ptr(c) for c in cols],
                                                 C.byref(h))
        else:
            Nz = N[2] if dim == 3 else 1
            create = lib.mfgpu_symbolic_create_full if full else lib.mfgpu_symbolic_create
            st = create(dim, N[0], N[1], Nz, width, max_side_length, C.byref(h))
        if st != _lib.MFGPU_OK:
            _raise(st, lib.mfgpu_symbolic_error().decode())
        self._h, self._lib = h, lib
        lv, nf, ns, nd = C.c_int(), C.c_int(), C.c_int(), C.c_int64()
        lib.mfgpu_symbolic_sizes(h, C.byref(lv), C.byref(nf), C.byref(ns), C.byref(nd))
        self.levels, self.n_fronts, self.n_seps, self.ndof = lv.value, nf.value, ns.value, nd.value

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.mfgpu_symbolic_destroy(self._h)
            self._h = None

    def front(self, f):
        lv, bx, n, m = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        p = C.POINTER(C.c_int)()
        st = self._lib.mfgpu_symbolic_front(self._h, f, C.byref(lv), C.byref(bx), C.byref(n),
                                            C.byref(m), C.byref(p))
        if st:
            raise IndexError(f)
        d = np.ctypeslib.as_array(p, shape=(n.value + m.value,)).copy() if n.value + m.value else \
            np.zeros(0, np.int32)
        off, ld = C.c_int64(), C.c_int()
        self._lib.mfgpu_symbolic_layout(self._h, 0, f, C.byref(off), C.byref(ld))
        return dict(level=lv.value, box=bx.value, n=n.value, m=m.value, dofs=d, off=off.value,
                    ld=ld.value)

    def sep(self, k):
        lv, ix, sz = C.c_int(), C.c_int(), C.c_int()
        p = C.POINTER(C.c_int)()
        boxes = (C.c_int * 2)()
        rows = (C.c_int * 2)()
        st = self._lib.mfgpu_symbolic_sep(self._h, k, C.byref(lv), C.byref(ix), C.byref(sz),
                                          C.byref(p), boxes, rows)
        if st:
            raise IndexError(k)
        d = np.ctypeslib.as_array(p, shape=(sz.value,)).copy() if sz.value else np.zeros(0, np.int32)
        off, ld = C.c_int64(), C.c_int()
        self._lib.mfgpu_symbolic_layout(self._h, 1, k, C.byref(off), C.byref(ld))
        return dict(level=lv.value, idx=ix.value, size=sz.value, dofs=d, boxes=list(boxes),
                    rows=list(rows), off=off.value, ld=ld.value)

    def dirty(self, modifiedDOFs):
        """(dirty flags per front, their flops) of a localized update."""
        mod = np.ascontiguousarray(sorted(set(int(d) for d in modifiedDOFs)), np.int32)
        out = np.zeros(self.n_fronts, np.uint8)
        fl = C.c_double()
        n = self._lib.mfgpu_symbolic_dirty(self._h, _lib._ptr(mod), len(mod), _lib._ptr(out),
                                           C.byref(fl))
        if n < 0:
            raise ValueError("modified DOF out of range")
        return out.astype(bool), fl.value

    def tasks(self, which):
        p = C.c_void_p()
        n = self._lib.mfgpu_symbolic_tasks(self._h, which, C.byref(p))
        if n <= 0:
            return np.zeros(0, TASK_DTYPE)
        buf = (C.c_char * (n * TASK_DTYPE.itemsize)).from_address(p.value)
        return np.frombuffer(bytes(buf), dtype=TASK_DTYPE)
