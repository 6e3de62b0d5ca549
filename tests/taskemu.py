"""Test helper: execute the product's assembly task tables with numpy.

The tables (mfgpu_symbolic_tasks) are what the device kernel k_tasks runs.
Feeding them the oracle's own child update matrices and separator blocks and
comparing the result with the oracle's assembled fronts proves the extend-add
maps bit for bit on the CPU, without a GPU.
"""
import numpy as np

ZERO, COPY, SPARSE, ADD = 0, 1, 2, 3


def arena_sizes(S):
    fe = 0
    for f in range(S.n_fronts):
        F = S.front(f)
        N = F["n"] + F["m"]
        fe = max(fe, F["off"] + F["ld"] * N + 1)
    se = 1
    for k in range(S.n_seps):
        s = S.sep(k)
        se = max(se, s["off"] + s["ld"] * s["size"] + 1)
    return fe, se


def run_tasks(tasks, arenas, A, dofs_table):
    """Apply task records to the two arenas (0: fronts, 1: separators)."""
    for t in tasks:
        R, Cn = int(t["rows"]), int(t["cols"])
        if R == 0 or Cn == 0:
            continue
        dst = arenas[int(t["dst_arena"])]
        dld, doff = int(t["dst_ld"]), int(t["dst_off"])
        ii, jj = np.meshgrid(np.arange(R), np.arange(Cn), indexing="ij")
        mask = (ii >= jj) if t["lower"] else np.ones_like(ii, bool)
        didx = doff + ii + jj * dld
        kind = int(t["kind"])
        if kind == ZERO:
            vals = np.zeros((R, Cn))
        elif kind in (COPY, ADD):
            src = arenas[int(t["src_arena"])]
            sld, soff = int(t["src_ld"]), int(t["src_off"])
            sidx = soff + (jj + ii * sld if t["trans"] else ii + jj * sld)
            vals = src[sidx]
        else:
            rd = dofs_table(int(t["row_dof"]), R)
            cd = dofs_table(int(t["col_dof"]), Cn)
            vals = A[rd][:, cd].toarray()
        if kind == ADD:
            dst[didx[mask]] = dst[didx[mask]] + vals[mask]
        else:
            dst[didx[mask]] = vals[mask]


class Emu:
    """Arena model keyed like the device layout of a Symbolic schedule."""

    def __init__(self, S, A):
        self.S = S
        self.A = A.tocsr()
        fe, se = arena_sizes(S)
        self.F = np.zeros(fe)
        self.SA = np.zeros(se)
        self.fronts = [S.front(f) for f in range(S.n_fronts)]
        self.seps = [S.sep(k) for k in range(S.n_seps)]
        # global DOF table: fronts then separators, as the schedule lays it out
        chunks = [F["dofs"] for F in self.fronts] + [s["dofs"] for s in self.seps]
        self.table = np.concatenate(chunks).astype(np.int64)
        self.ftasks = S.tasks(0)
        self.stasks = S.tasks(1)
        self.atasks = S.tasks(2)

    def dofs(self, off, count):
        return self.table[off:off + count]

    def block(self, f):
        """Dense symmetric copy of front f's lower triangle."""
        F = self.fronts[f]
        N, ld, off = F["n"] + F["m"], F["ld"], F["off"]
        M = self.F[off:off + ld * N].reshape(N, ld).T[:N, :N].copy()
        L = np.tril(M)
        return L + np.tril(L, -1).T

    def set_block(self, f, M):
        F = self.fronts[f]
        N, ld, off = F["n"] + F["m"], F["ld"], F["off"]
        view = self.F[off:off + ld * N].reshape(N, ld).T
        view[:N, :N] = np.tril(M)

    def block_full(self, f):
        """Front f as stored (both triangles; full-storage tables)."""
        F = self.fronts[f]
        N, ld, off = F["n"] + F["m"], F["ld"], F["off"]
        return self.F[off:off + ld * N].reshape(N, ld).T[:N, :N].copy()

    def set_block_full(self, f, M):
        F = self.fronts[f]
        N, ld, off = F["n"] + F["m"], F["ld"], F["off"]
        self.F[off:off + ld * N].reshape(N, ld).T[:N, :N] = M

    def sep_block(self, k):
        s = self.seps[k]
        n, ld, off = s["size"], s["ld"], s["off"]
        M = self.SA[off:off + ld * n].reshape(n, ld).T[:n, :n].copy()
        L = np.tril(M)
        return L + np.tril(L, -1).T

    def set_sep(self, k, M):
        s = self.seps[k]
        n, ld, off = s["size"], s["ld"], s["off"]
        view = self.SA[off:off + ld * n].reshape(n, ld).T
        view[:n, :n] = np.tril(M)

    def run(self, tasks, owners=None):
        sel = tasks if owners is None else tasks[np.isin(tasks["owner"], owners)]
        run_tasks(sel, [self.F, self.SA], self.A, self.dofs)

    def level_fronts(self, ell):
        return [f for f, F in enumerate(self.fronts) if F["level"] == ell]

    def level_seps(self, ell):
        return [k for k, s in enumerate(self.seps) if s["level"] == ell]
