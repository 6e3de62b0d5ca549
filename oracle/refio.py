"""Test infrastructure: read/write the binary files exchanged with the reference
harness (oracle/ref_harness.cpp).  Nothing in the product imports this module.

Input file layout (little endian), consumed by readInput() in ref_harness.cpp:
  int32[12]  dim, Nx, Ny, Nz, width, maxSide, dumpSymbolic, dumpFronts,
             doUpdate, nrhs, timeReps, solveReps
  float64[3] hx, hy, hz
  float64[]  coefficient field 1, C order of the reference's A[i][j](k)
             (shape (Nx+2w, Ny+2w[, Nz+2w]))
  float64[]  coefficient field 2 (only when doUpdate)
  float64[]  nrhs right-hand sides of length n, one after the other

Output file: a stream of records  uint32 name_len, name, char dtype ('i'|'d'),
uint64 count, payload.
"""
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "ref_harness")


def have_reference():
    return os.path.isfile(REF_BIN) and os.access(REF_BIN, os.X_OK)


def write_input(path, dim, N, width, max_side, coef1, coef2=None, rhs=None,
                h=(1.0, 1.0, 1.0), dump_symbolic=1, dump_fronts=0,
                time_reps=0, solve_reps=0):
    Nx, Ny = N[0], N[1]
    Nz = N[2] if dim == 3 else 1
    rhs = np.zeros((0,)) if rhs is None else np.atleast_2d(np.asarray(rhs, np.float64))
    nrhs = 0 if rhs.size == 0 else rhs.shape[0]
    hdr = np.array([dim, Nx, Ny, Nz, width, max_side, dump_symbolic, dump_fronts,
                    1 if coef2 is not None else 0, nrhs, time_reps, solve_reps],
                   dtype=np.int32)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.asarray(h, np.float64).tobytes())
        f.write(np.ascontiguousarray(coef1, np.float64).tobytes())
        if coef2 is not None:
            f.write(np.ascontiguousarray(coef2, np.float64).tobytes())
        if nrhs:
            f.write(np.ascontiguousarray(rhs, np.float64).tobytes())


def read_records(path):
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        (nl,) = struct.unpack_from("<I", data, pos)
        pos += 4
        name = data[pos:pos + nl].decode()
        pos += nl
        dt = chr(data[pos])
        pos += 1
        (cnt,) = struct.unpack_from("<Q", data, pos)
        pos += 8
        es = 8 if dt == "d" else 4
        arr = np.frombuffer(data, dtype=np.float64 if dt == "d" else np.int32,
                            count=cnt, offset=pos).copy()
        pos += es * cnt
        out[name] = arr
    # Fold "X.shape" records into 2D column-major matrices.
    for k in [k for k in out if k.endswith(".shape")]:
        base = k[:-6]
        m, n = int(out[k][0]), int(out[k][1])
        v = out.get(base)
        if v is not None and v.size == m * n:
            out[base] = v.reshape((n, m)).T.copy()
        else:
            out[base] = np.zeros((m, n))
        del out[k]
    return out


def run_reference(workdir, dim, N, width, max_side, coef1, coef2=None, rhs=None,
                  h=(1.0, 1.0, 1.0), dump_symbolic=1, dump_fronts=0, timeout=3600, threads=None):
    """Run the compiled reference once and return its records (BLAS threads:
    `threads`, else OPENBLAS_NUM_THREADS from the environment, else 1)."""
    os.makedirs(workdir, exist_ok=True)
    inp = os.path.join(workdir, "in.bin")
    outp = os.path.join(workdir, "out.bin")
    write_input(inp, dim, N, width, max_side, coef1, coef2, rhs, h,
                dump_symbolic, dump_fronts)
    env = dict(os.environ)
    if threads is not None:
        env["OPENBLAS_NUM_THREADS"] = str(threads)
    env.setdefault("OPENBLAS_NUM_THREADS", "1")
    subprocess.run([REF_BIN, "dump", inp, outp], check=True, env=env, timeout=timeout)
    return read_records(outp)


def reference_csr(workdir, dim, N, width, coef, h=(1.0, 1.0, 1.0)):
    """CSR built by the reference fixture only (test_include/DE/buildLaplacian.hpp)."""
    os.makedirs(workdir, exist_ok=True)
    inp = os.path.join(workdir, "csr_in.bin")
    outp = os.path.join(workdir, "csr_out.bin")
    write_input(inp, dim, N, width, 1, coef, None, None, h, 0, 0)
    subprocess.run([REF_BIN, "csr", inp, outp], check=True, timeout=600)
    return read_records(outp)


def time_reference(workdir, dim, N, width, max_side, coef1, coef2=None, rhs=None,
                   h=(1.0, 1.0, 1.0), reps=1, solve_reps=1, threads=None, timeout=3600):
    """Time the reference's Factor / Update / Solve; returns the parsed JSON."""
    import json
    os.makedirs(workdir, exist_ok=True)
    inp = os.path.join(workdir, "time_in.bin")
    write_input(inp, dim, N, width, max_side, coef1, coef2, rhs, h, 0, 0,
                time_reps=reps, solve_reps=solve_reps)
    env = dict(os.environ)
    if threads is not None:
        env["OPENBLAS_NUM_THREADS"] = str(threads)
    p = subprocess.run([REF_BIN, "time", inp, "/dev/null"], check=True, env=env,
                       capture_output=True, text=True, timeout=timeout)
    return json.loads(p.stdout.strip().splitlines()[-1])
