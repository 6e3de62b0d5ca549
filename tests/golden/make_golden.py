"""Generate the golden fixtures in this directory by running the reference
itself (oracle/_ref/ref_harness, compiled from the reference sources by
oracle/Makefile) on small seeded problems.

Each fixture <case>.npz holds what the reference computed:
  csr_sha256            hash of the reference-built CSR (row_ptr, col_ind, val)
  levels                tree depth
  box_<l>_int / _bd     concatenated Box::intDOFs / bdDOFs of level l, with
  box_<l>_int_ptr / ...  offsets per box (include/DE/mf.hpp:45-55)
  sep_<l> / sep_<l>_ptr concatenated Edge/Face::DOFs of level l
  rhs, solve, apply, resid          one right-hand side and the reference's results
  moddofs, upd_solve, upd_resid     after Update() with a 5-cell patch x10
  (2D 31x31 only) per-front S and A11post of the levels >= 1

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "updating-multifrontal_b200"))

import refio  # noqa: E402
from mfgpu import stencil  # noqa: E402

CASES = {
    "2d_31x31_m4": dict(dim=2, N=(31, 31), ms=4, coef="logu", fronts=True),
    "2d_23x57_m4": dict(dim=2, N=(23, 57), ms=4, coef="logu", fronts=False),
    "2d_130x70_m4": dict(dim=2, N=(130, 70), ms=4, coef="logu", fronts=False),
    "2d_127x127_m8_uniform": dict(dim=2, N=(127, 127), ms=8, coef="uniform", fronts=False),
    "3d_15x15x15_m4": dict(dim=3, N=(15, 15, 15), ms=4, coef="logu", fronts=False),
    "3d_13x17x11_m3": dict(dim=3, N=(13, 17, 11), ms=3, coef="logu", fronts=False),
}
SEED = 20261203


def csr_hash(rp, ci, val):
    h = hashlib.sha256()
    for a in (np.asarray(rp, np.int32), np.asarray(ci, np.int32), np.asarray(val, np.float64)):
        h.update(a.tobytes())
    return h.hexdigest()


def inputs(case, i):
    N = case["N"]
    if case["coef"] == "uniform":
        a1 = stencil.uniform_coefficients(N)
    else:
        a1 = stencil.loguniform_coefficients(N, 0.1, 10.0, SEED + 100 + i)
    a2 = stencil.scale_box(a1, [2] * len(N), 5, 10.0)
    n = int(np.prod(N))
    rhs = stencil.uniform_rhs(n, 1, SEED + 200 + i)
    return a1, a2, rhs


def flatten(lists):
    ptr = np.zeros(len(lists) + 1, np.int64)
    for k, l in enumerate(lists):
        ptr[k + 1] = ptr[k] + len(l)
    data = np.concatenate([np.asarray(l, np.int32) for l in lists]) if lists else np.zeros(0, np.int32)
    return data.astype(np.int32), ptr


def main():
    if not refio.have_reference():
        sys.exit("oracle/_ref/ref_harness is not built (run make in oracle/)")
    for i, (name, case) in enumerate(sorted(CASES.items())):
        a1, a2, rhs = inputs(case, i)
        with tempfile.TemporaryDirectory() as d:
            R1 = refio.run_reference(d, case["dim"], case["N"], 1, case["ms"], a1, None, rhs,
                                     dump_fronts=1 if case["fronts"] else 0)
            R2 = refio.run_reference(d, case["dim"], case["N"], 1, case["ms"], a1, a2, rhs,
                                     dump_symbolic=0)
        out = {"csr_sha256": np.array(csr_hash(R1["A1.row_ptr"], R1["A1.col_ind"], R1["A1.val"])),
               "levels": np.array(int(R1["levels"][0]))}
        L = int(R1["levels"][0])
        for ell in range(L):
            nb = len([k for k in R1 if k.startswith(f"box.{ell}.") and k.endswith(".int")])
            ints = [R1[f"box.{ell}.{b}.int"] for b in range(nb)]
            bds = [R1[f"box.{ell}.{b}.bd"] for b in range(nb)]
            out[f"box_{ell}_int"], out[f"box_{ell}_int_ptr"] = flatten(ints)
            out[f"box_{ell}_bd"], out[f"box_{ell}_bd_ptr"] = flatten(bds)
            if ell >= 1:
                ns = len([k for k in R1 if k.startswith(f"sep.{ell}.") and k.endswith(".dofs")])
                out[f"sep_{ell}"], out[f"sep_{ell}_ptr"] = flatten([R1[f"sep.{ell}.{e}.dofs"]
                                                                    for e in range(ns)])
            if case["fronts"] and ell >= 1:
                for b in range(nb):
                    out[f"S_{ell}_{b}"] = R1[f"box.{ell}.{b}.S"]
                    out[f"A11post_{ell}_{b}"] = R1[f"box.{ell}.{b}.A11post"]
        out["rhs"] = rhs[0]
        out["solve"] = R1["f1.solve.0"]
        out["apply"] = R1["f1.apply.0"]
        out["resid"] = R1["f1.resid.0"]
        out["moddofs"] = R2["moddofs"]
        out["upd_solve"] = R2["f2.solve.0"]
        out["upd_resid"] = R2["f2.resid.0"]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "levels", L, "resid", float(R1["f1.resid.0"][0]))


if __name__ == "__main__":
    main()
