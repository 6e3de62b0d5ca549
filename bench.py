#!/usr/bin/env python3
"""Benchmark: factor + localized update + solve on one B200 per rank, mixed
precision against FP64.

Workload (default, `3d-127`): 3D 7-point variable-coefficient Laplacian on a
127 x 127 x 127 interior grid (n = 2,048,383), node coefficients iid
log-uniform in [0.1, 100] from a fixed seed, leaf parameter 4 (leaf boxes of
7 x 7 x 7 cells), one right-hand side iid uniform[-1, 1].  One step is
  1. a full factorization of the matrix (values resident in HBM),
  2. a localized update: coefficients x10 on a 9 x 9 x 9-cell patch at a
     seeded position, refactoring only the root paths of the leaves it touches,
  3. a solve with the updated factorization,
in mixed precision: FP32 factorization of the diagonally scaled matrix with
the Schur-complement updates of the large-front levels on the tensor cores
(three-term TF32 products), then conjugate gradients in FP64 preconditioned by
it until ||b - A x|| / ||b|| <= 1e-10.  `value` is the algorithmic TFLOP/s of
that step: Cholesky-form flops sum(n^3/3 + n^2 m + n m^2) over the factored
fronts, the same over the fronts the update refactors, and 2(n^2 + 2nm) per
front and right-hand side for the solve, over the device time of the step.
`precision_comparison` times the FP64 path on the same workload and step, and
gives the forward error of the mixed solution against the FP64 one.

`--impl reference` times the reference's own CPU implementation
(oracle/_ref/ref_harness, compiled from the reference sources) on the host
cores with every host thread, on a bounded sample of the workload (for
3d-127: the octant [0, 63)^3 of the same coefficient field, whose tree is one
of the eight level-1 subtrees; the full grid needs about 171 GB of host memory
and tens of minutes per sample), with the work counted from the reference's
own front sizes.  That arm imports nothing from the product.

Multi-GPU: the path does not shard (one problem per GPU); N ranks run N
independent replicas ("weak" scaling) and `value` is the aggregate.
"""
import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "updating-multifrontal_b200")


def _load_stencil():
    """The stencil builder (plain numpy) loaded by file, so that the reference
    arm touches no module of the product package."""
    spec = importlib.util.spec_from_file_location(
        "mf_bench_stencil", os.path.join(PKG, "mfgpu", "stencil.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


stencil = _load_stencil()

SEED0 = 20261203
METRIC = "factor+update+solve s & TFLOP/s: mixed vs FP64 on 1 B200 at resid ≤1e-10; p99"
WORKLOADS = {
    # the 3D workload: log-uniform [0.1, 100], leaf parameter 4, one RHS; the
    # reference arm and the CPU baseline time the octant [0, 63)^3
    "3d-127": dict(dim=3, N=(127, 127, 127), max_side=4, lo=0.1, hi=100.0, nrhs=1, patch=9,
                   factor=10.0, seed=SEED0 + 3, sample_octant=63, ref_steps=2,
                   label="3D 127^3 7-point, a log-U[0.1,100], leaf 7^3 (maxSideLength 4), 1 RHS, "
                         "9^3 patch x10 update"),
    # the 2D variable-coefficient workload with 4 right-hand sides
    "2d-1023": dict(dim=2, N=(1023, 1023), max_side=8, lo=0.1, hi=10.0, nrhs=4, patch=9,
                    factor=10.0, seed=SEED0 + 2, ref_steps=20,
                    label="2D 1023^2 5-point, a log-U[0.1,10], leaf 15^2 (maxSideLength 8), 4 RHS, "
                          "9^2 patch x10 update"),
    # the CPU-runnable 2D workload (a = 1, leaf parameter 4, one RHS)
    "2d-127": dict(dim=2, N=(127, 127), max_side=4, lo=1.0, hi=1.0, nrhs=1, patch=9,
                   factor=10.0, seed=SEED0 + 1, ref_steps=20,
                   label="2D 127^2 5-point, a = 1, leaf 7^2 (maxSideLength 4), 1 RHS, "
                         "9^2 patch x10 update"),
    # 256 independent 2D problems in one handle (sides 63..511, 1-8 RHS each)
    "batch256": dict(batch=True, count=256, sides=(63, 127, 255, 511), max_side=4, lo=0.1, hi=10.0,
                     max_nrhs=8, seed=SEED0 + 5),
    # update serving on a resident 3D 95^3 factorization: Poisson arrivals, each
    # request a coefficient box (side 3-15, factor log-U[0.1,10]) + 1-16 RHS
    "serve95": dict(serve=True, dim=3, N=(95, 95, 95), max_side=4, lo=0.1, hi=10.0, side=(3, 15),
                    nrhs=(1, 16), seed=SEED0 + 6),
    # a smaller 3D case of the same kind (profiling captures, quick checks)
    "3d-63": dict(dim=3, N=(63, 63, 63), max_side=4, lo=0.1, hi=100.0, nrhs=1, patch=5,
                  factor=10.0, seed=SEED0 + 4, ref_steps=4,
                  label="3D 63^3 7-point, a log-U[0.1,100], leaf 7^3 (maxSideLength 4), 1 RHS, "
                        "5^3 patch x10 update"),
}


def make_problem(w, rank=0):
    """Coefficients before / after the update, both CSR matrices, the modified
    DOFs, the right-hand sides (nrhs, n) and the patch corner."""
    N = w["N"]
    seed = w["seed"] + 1000 * rank
    if w["lo"] == w["hi"]:
        a1 = stencil.uniform_coefficients(N, value=w["lo"])
    else:
        a1 = stencil.loguniform_coefficients(N, w["lo"], w["hi"], seed)
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    lo = [int(rng.integers(0, n - w["patch"] + 1)) for n in N]
    a2 = stencil.scale_box(a1, lo, w["patch"], w["factor"])
    A1 = stencil.build_laplacian(a1)
    A2 = stencil.build_laplacian(a2)
    mod = stencil.modified_dofs(A1, A2)
    b = stencil.uniform_rhs(A1.n, w["nrhs"], seed + 11)
    return a1, a2, A1, A2, mod, b, lo


def reference_sample(w):
    """The bounded CPU sample of a workload for the reference: (dim, N,
    coefficients before / after the update, rhs (nrhs, n), description).  For
    3d-127 the octant [0, s)^3 of the workload's coefficient field (cells
    0..s-1 are nodes 1..s, plus the boundary nodes 0 and s+1), its patch moved
    into the octant; otherwise the whole workload."""
    a1, a2, A1, A2, mod, b, lo = make_problem(w)
    s = w.get("sample_octant")
    if not s:
        return w["dim"], w["N"], a1, a2, b, "the full workload"
    sub = a1[tuple(slice(0, s + 2) for _ in range(w["dim"]))].copy()
    lo_s = [l % (s - w["patch"] + 1) for l in lo]
    sub2 = stencil.scale_box(sub, lo_s, w["patch"], w["factor"])
    Ns = tuple([s] * w["dim"])
    n = s ** w["dim"]
    bs = stencil.uniform_rhs(n, w["nrhs"], w["seed"] + 11)
    desc = (f"the octant [0,{s})^{w['dim']} of the workload's coefficient field ({n} unknowns, "
            f"one of the eight level-1 subtrees of the 127^3 tree), its {w['patch']}^{w['dim']} "
            f"patch x{w['factor']:g} moved to {lo_s}")
    return w["dim"], Ns, sub, sub2, bs, desc


def reference_time(dim, N, max_side, a1, a2, b, threads, reps, timeout=3000):
    """Run the compiled reference (oracle/_ref) in timing mode; returns its JSON
    (seconds per call and the work figures from its own front sizes), or None
    when the harness is not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refio
    if not refio.have_reference():
        return None
    with tempfile.TemporaryDirectory() as d:
        return refio.time_reference(d, dim, N, 1, max_side, a1, a2, b, reps=reps, solve_reps=1,
                                    threads=threads, timeout=timeout)


def ref_step_flops(res, nrhs):
    return res["factor_flops"] + res["update_flops"] + nrhs * res["solve_flops_per_rhs"]


def cpu_info():
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    mem_gb = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemTotal:"):
                    mem_gb = round(int(line.split()[1]) / 2 ** 20, 1)
    except OSError:
        pass
    return model, os.cpu_count() or 1, mem_gb


def solve_flops(fronts_nm, nrhs):
    return nrhs * sum(2.0 * (n * n + 2.0 * n * m) for n, m in fronts_nm)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def measured_gemm_peak(torch, dtype):
    """cuBLAS GEMM throughput (torch matmul, 8192^3, TF32 off), best of 5, TFLOP/s."""
    n = 8192
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.isfile(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def whole_job(local_ms, local_flops, device):
    """Replicas on N ranks: the job's time is the slowest rank's (max over
    ranks) and its work the sum of every rank's algorithmic flops.  Returns
    (TFLOP/s of the whole job, max ms, total flops); every rank gets the same
    values.  One rank: its own."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    f = torch.tensor([float(local_flops)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(f, op=dist.ReduceOp.SUM)
    ms, fl = float(t.item()), float(f.item())
    return fl / (ms * 1e-3) / 1e12, ms, fl


def pct(v, q):
    return float(np.percentile(np.asarray(v, np.float64), q))


def dtype_of(precision):
    return "f64" if precision == "fp64" else \
        "f32 factor (tf32x3 tensor-core Schur updates) + f64 residual/refinement"


def config_of(w, args, precision):
    return {"workload": f"{args.workload} ({w['label']})", "grid": list(w["N"]),
            "max_side_length": w["max_side"], "nrhs": w["nrhs"], "precision": precision,
            "parallelism": f"replicas x{args.gpus}",
            "l2": "inputs larger than L2 (front arena > 126 MB); no flush needed"}


# ---------------------------------------------------------------------------
# reference arm: the reference's CPU code only, nothing of the product
# ---------------------------------------------------------------------------
def run_reference_arm(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if w.get("batch"):
        return run_reference_arm_batch(args, w)
    dim, N, a1, a2, b, desc = reference_sample(w)
    threads = os.cpu_count() or 1
    warm = 1
    steps = max(1, min(args.steps, w.get("ref_steps", args.steps)))
    res = reference_time(dim, N, w["max_side"], a1, a2, b, threads, reps=warm + steps)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference harness oracle/_ref/ref_harness not built"}))
        return 0
    model, _, mem = cpu_info()
    tf, tu, ts = res["factor_s"][warm:], res["update_s"][warm:], res["solve_s"][warm:]
    step_s = [tf[i] + tu[i] + ts[i] for i in range(len(tf))]
    us = [tu[i] + ts[i] for i in range(len(tf))]
    fl = ref_step_flops(res, w["nrhs"])
    t = statistics.median(step_s)
    value = fl / t / 1e12
    cfg = config_of(w, args, args.precision)
    cfg["sample"] = desc
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s",
        "n_gpus": args.gpus, "steps": len(step_s), "warmup": warm, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded coefficients and right-hand sides)", "config": cfg,
        "phases_s": {"factor_p50": statistics.median(tf), "update_p50": statistics.median(tu),
                     "solve_p50": statistics.median(ts), "step_p50": t, "step_p99": pct(step_s, 99),
                     "update_solve_p50": statistics.median(us), "update_solve_p99": pct(us, 99)},
        "flops_per_step": {"factor": res["factor_flops"], "update": res["update_flops"],
                           "solve": w["nrhs"] * res["solve_flops_per_rhs"],
                           "counted_from": "the reference's own front sizes (intDOFs, bdDOFs)"},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(step_s)} x (factor + update + {w['nrhs']}-RHS solve) of "
                                   f"{desc}, OPENBLAS_NUM_THREADS={threads}",
                         "cpu": model, "host_mem_gb": mem},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_reference_arm_batch(args, w):
    """Reference arm of a batch workload: the reference factors and solves one
    problem per object, so each sample runs the batch's members one at a time
    (from the first) for about 20 s; value = their algorithmic flops / time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refio
    if not refio.have_reference():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference harness oracle/_ref/ref_harness not built"}))
        return 0
    members = make_batch(w)
    threads = os.cpu_count() or 1
    samples = []
    warm = 1
    for rep in range(warm + max(1, min(args.steps, 4))):
        t_tot, fl_tot, used = 0.0, 0.0, 0
        for dim, N, ms, a, A, b in members:
            if t_tot > 20.0:
                break
            with tempfile.TemporaryDirectory() as d:
                res = refio.time_reference(d, dim, N, 1, ms, a, None, b, reps=1, solve_reps=1,
                                           threads=threads)
            t_tot += res["factor_s"][0] + res["solve_s"][0]
            fl_tot += res["factor_flops"] + b.shape[0] * res["solve_flops_per_rhs"]
            used += 1
        if rep >= warm:
            samples.append((t_tot, fl_tot, used))
    vals = [fl / t / 1e12 for t, fl, _ in samples]
    value = statistics.median(vals)
    model, _, mem = cpu_info()
    t_med = statistics.median([t for t, _, _ in samples])
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s",
        "n_gpus": args.gpus, "steps": len(samples), "warmup": warm, "ms_per_step": t_med * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded coefficients and right-hand sides)",
        "config": {"workload": args.workload, "precision": args.precision,
                   "sample": f"first {samples[0][2]} of {len(members)} problems per step"},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads, "kind": "reference",
                         "sample": f"factor + solve of the first {samples[0][2]} batch members, "
                                   f"one at a time, OPENBLAS_NUM_THREADS={threads}", "cpu": model,
                         "host_mem_gb": mem},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def front_sizes(w):
    from mfgpu import Symbolic
    S = Symbolic(w["dim"], w["N"], 1, w["max_side"])
    return [(S.front(f)["n"], S.front(f)["m"]) for f in range(S.n_fronts)]


def update_flops(w, mod):
    """Flops of the fronts a localized update refactors (root paths of dirty leaves)."""
    from mfgpu import Symbolic
    S = Symbolic(w["dim"], w["N"], 1, w["max_side"])
    return S.dirty(mod)[1]


class SingleWork:
    """One problem: step = full factorization + localized update + solve."""

    def __init__(self, w, rank, local, prec, problem=None):
        from mfgpu import MF2D, MF3D
        self.w = w
        self.a1, self.a2, self.A1, self.A2, self.mod, self.b, _ = problem or make_problem(w, rank)
        self.n, self.nnz, self.nrhs = self.A1.n, self.A1.nnz, w["nrhs"]
        N = w["N"]
        if w["dim"] == 2:
            self.F = MF2D(self.A1, N[0], N[1], 1, w["max_side"], device=local, precision=prec)
        else:
            self.F = MF3D(self.A1, N[0], N[1], N[2], 1, w["max_side"], device=local,
                          precision=prec)
        self.fl = front_sizes(w)
        self.upd_fl = update_flops(w, self.mod)

    def to_device(self, torch):
        self.dv1 = torch.from_numpy(self.A1.val).to("cuda")
        self.dv2 = torch.from_numpy(self.A2.val).to("cuda")
        self.db = torch.from_numpy(np.ascontiguousarray(self.b)).to("cuda")   # column-major n x nrhs
        self.dx = torch.empty_like(self.db)

    def step(self, marks=None):
        """One step; `marks` (three events) are recorded after the factor, the
        update and the solve on the handle's stream."""
        F = self.F
        F.refactor_device(self.dv1.data_ptr(), self.nnz)
        if marks:
            marks[0].record(self.stream)
        F.update_device(self.dv2.data_ptr(), self.nnz, self.mod)
        if marks:
            marks[1].record(self.stream)
        F.solve_device(self.db.data_ptr(), self.dx.data_ptr(), self.nrhs, self.n)
        if marks:
            marks[2].record(self.stream)

    def solution(self):
        return self.dx.cpu().numpy()          # (nrhs, n)

    def resid(self):
        x = self.solution()
        return max(float(np.linalg.norm(self.A2.matvec(x[r]) - self.b[r]) /
                         np.linalg.norm(self.b[r])) for r in range(self.nrhs))

    def flops_breakdown(self):
        return {"factor": self.F.info()["factor_flops"], "update": self.upd_fl,
                "solve": solve_flops(self.fl, self.nrhs)}

    def step_flops(self):
        return sum(self.flops_breakdown().values())

    def e2e_setup(self, torch):
        self.hv1 = torch.from_numpy(self.A1.val).pin_memory()
        self.hv2 = torch.from_numpy(self.A2.val).pin_memory()
        self.hb = torch.from_numpy(np.ascontiguousarray(self.b)).pin_memory()
        self.hx = torch.empty_like(self.hb).pin_memory()
        self.mod32 = np.ascontiguousarray(self.mod, np.int32)

    def e2e_step(self):
        F = self.F
        F.refactor_host_ptr(self.hv1.data_ptr(), self.nnz)
        F.update_host_ptr(self.hv2.data_ptr(), self.nnz, self.mod32)
        F.solve_host_ptr(self.hb.data_ptr(), self.hx.data_ptr(), self.nrhs, self.n)

    def e2e_bytes(self):
        return (2 * self.nnz * 8 + self.n * self.nrhs * 8 + self.mod32.size * 4,
                self.n * self.nrhs * 8)

    def config(self, args, precision):
        return config_of(self.w, args, precision)

    def cpu_baseline(self, threads):
        dim, N, a1, a2, b, desc = reference_sample(self.w)
        res = reference_time(dim, N, self.w["max_side"], a1, a2, b, threads, reps=1)
        if res is None:
            return None
        tcpu = res["factor_s"][0] + res["update_s"][0] + res["solve_s"][0]
        model, _, mem = cpu_info()
        return {"value": ref_step_flops(res, self.nrhs) / tcpu / 1e12, "unit": "TFLOP/s",
                "cores": threads, "kind": "reference",
                "sample": f"1 x (factor + update + {self.nrhs}-RHS solve) of {desc} "
                          f"({tcpu:.2f} s), OPENBLAS_NUM_THREADS={threads}",
                "update_solve_s": res["update_s"][0] + res["solve_s"][0],
                "cpu": model, "host_mem_gb": mem}


def make_batch(w, rank=0):
    """The batch members: (dim, N, maxSideLength, coefficients, CSR, rhs (k, n))."""
    seed = w["seed"] + 1000 * rank
    rng = np.random.Generator(np.random.PCG64(seed))
    sides = rng.choice(np.asarray(w["sides"]), size=w["count"])
    ks = rng.integers(1, w["max_nrhs"] + 1, size=w["count"])
    out = []
    for i, (side, k) in enumerate(zip(sides, ks)):
        N = (int(side), int(side))
        a = stencil.loguniform_coefficients(N, w["lo"], w["hi"], seed + 1 + i)
        A = stencil.build_laplacian(a)
        b = stencil.uniform_rhs(A.n, int(k), seed + 100000 + i)
        out.append((2, N, w["max_side"], a, A, b))
    return out


class BatchWork:
    """Independent problems in one handle: step = factorization of every
    problem + one solve with every problem's right-hand sides."""

    def __init__(self, w, rank, local, prec, problem=None):
        from mfgpu import MFBatch, Symbolic
        self.w = w
        self.members = make_batch(w, rank)
        self.F = MFBatch([(A, N, 1, ms) for dim, N, ms, a, A, b in self.members], device=local,
                         precision=prec)
        self.A = self.F.A
        self.n, self.nnz = self.A.n, self.A.nnz
        self.nrhs = max(b.shape[0] for *_, b in self.members)
        self.B = self.F.join([b.T for *_, b in self.members], self.nrhs)
        self.factor_fl = self.F.info()["factor_flops"]
        self.solve_fl = 0.0
        cache = {}
        for dim, N, ms, a, A, b in self.members:
            if N not in cache:
                Sp = Symbolic(dim, N, 1, ms)
                cache[N] = [(Sp.front(f)["n"], Sp.front(f)["m"]) for f in range(Sp.n_fronts)]
            self.solve_fl += solve_flops(cache[N], b.shape[0])

    def to_device(self, torch):
        self.dv = torch.from_numpy(self.A.val).to("cuda")
        self.db = torch.from_numpy(np.ascontiguousarray(self.B.T)).to("cuda")   # (nrhs, n)
        self.dx = torch.empty_like(self.db)

    def step(self, marks=None):
        self.F.refactor_device(self.dv.data_ptr(), self.nnz)
        if marks:
            marks[0].record(self.stream)
            marks[1].record(self.stream)
        self.F.solve_device(self.db.data_ptr(), self.dx.data_ptr(), self.nrhs, self.n)
        if marks:
            marks[2].record(self.stream)

    def solution(self):
        return self.dx.cpu().numpy()

    def resid(self):
        X = self.solution().T
        worst = 0.0
        for (dim, N, ms, a, A, b), x in zip(self.members, self.F.split(X)):
            for c in range(b.shape[0]):
                worst = max(worst, float(np.linalg.norm(A.matvec(x[:, c]) - b[c]) /
                                         np.linalg.norm(b[c])))
        return worst

    def flops_breakdown(self):
        return {"factor": self.factor_fl, "update": 0.0, "solve": self.solve_fl}

    def step_flops(self):
        return self.factor_fl + self.solve_fl

    def e2e_setup(self, torch):
        self.hv = torch.from_numpy(self.A.val).pin_memory()
        self.hb = torch.from_numpy(np.ascontiguousarray(self.B.T)).pin_memory()
        self.hx = torch.empty_like(self.hb).pin_memory()

    def e2e_step(self):
        self.F.refactor_host_ptr(self.hv.data_ptr(), self.nnz)
        self.F.solve_host_ptr(self.hb.data_ptr(), self.hx.data_ptr(), self.nrhs, self.n)

    def e2e_bytes(self):
        return self.nnz * 8 + self.n * self.nrhs * 8, self.n * self.nrhs * 8

    def config(self, args, precision):
        sides = [N[0] for _, N, *_ in self.members]
        return {"workload": f"{args.workload} ({self.w['count']} 2D 5-point problems, sides from "
                            f"{sorted(set(self.w['sides']))}, a log-U[{self.w['lo']},{self.w['hi']}], "
                            f"maxSideLength {self.w['max_side']}, 1-{self.w['max_nrhs']} RHS each; "
                            "step = factor + solve of every problem)",
                "problems": len(self.members), "ndof": self.n,
                "sides_count": {str(s): sides.count(s) for s in sorted(set(sides))},
                "nrhs_total": int(sum(b.shape[0] for *_, b in self.members)),
                "precision": precision, "parallelism": f"replicas x{args.gpus}",
                "l2": "inputs larger than L2 (front arena > 126 MB); no flush needed"}

    def cpu_baseline(self, threads):
        # the reference on the batch's first members, one at a time, about 20 s
        t_tot, fl_tot, used = 0.0, 0.0, 0
        for dim, N, ms, a, A, b in self.members:
            if t_tot > 20.0:
                break
            res = reference_time(dim, N, ms, a, None, b, threads, reps=1)
            if res is None:
                return None
            t_tot += res["factor_s"][0] + res["solve_s"][0]
            fl_tot += res["factor_flops"] + b.shape[0] * res["solve_flops_per_rhs"]
            used += 1
        model, _, mem = cpu_info()
        return {"value": fl_tot / t_tot / 1e12, "unit": "TFLOP/s", "cores": threads,
                "kind": "reference",
                "sample": f"factor + solve of the first {used} batch members one at a time "
                          f"({t_tot:.2f} s), OPENBLAS_NUM_THREADS={threads}", "cpu": model,
                "host_mem_gb": mem}


def timed_steps(torch, work, steps):
    """`steps` steps on the work's stream; returns (total ms, per-step ms, per
    step (factor, update, solve) ms)."""
    st = work.stream
    with torch.cuda.stream(st):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        rec = []
        for _ in range(steps):
            s0 = torch.cuda.Event(enable_timing=True)
            marks = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            s0.record(st)
            work.step(marks)
            rec.append((s0, marks))
        e1.record(st)
    st.synchronize()
    per = [s0.elapsed_time(m[2]) for s0, m in rec]
    phases = [(s0.elapsed_time(m[0]), m[0].elapsed_time(m[1]), m[1].elapsed_time(m[2]))
              for s0, m in rec]
    return e0.elapsed_time(e1), per, phases


def phase_stats(per, phases):
    us = [u + s for _, u, s in phases]
    return {"step_ms_p50": statistics.median(per), "step_ms_p99": pct(per, 99),
            "factor_ms_p50": statistics.median(p[0] for p in phases),
            "update_ms_p50": statistics.median(p[1] for p in phases),
            "solve_ms_p50": statistics.median(p[2] for p in phases),
            "update_solve_ms_p50": statistics.median(us), "update_solve_ms_p99": pct(us, 99)}


def forward_error(x, ref):
    """max over right-hand sides of ||x - ref|| / ||ref|| (rows = right-hand sides)."""
    return max(float(np.linalg.norm(x[r] - ref[r]) / np.linalg.norm(ref[r]))
               for r in range(ref.shape[0]))


def other_precision_run(torch, w, rank, local, prec, args, problem):
    """The other precision on the same workload and step, with a bounded number
    of timed steps (its handle is created after the first one was released)."""
    Work = BatchWork if w.get("batch") else SingleWork
    w2 = Work(w, rank, local, prec, problem)
    w2.stream = torch.cuda.Stream()
    w2.F.set_stream(w2.stream.cuda_stream)
    w2.to_device(torch)
    if args.autotune > 0:
        w2.F.autotune(args.autotune)
    for _ in range(3):
        w2.step()
    torch.cuda.synchronize()
    steps = max(1, min(args.steps, args.compare_steps))
    ms, per, phases = timed_steps(torch, w2, steps)
    out = {"steps": steps, "warmup": 3, "ms_per_step": ms / steps,
           "value": w2.step_flops() * steps / (ms * 1e-3) / 1e12}
    out.update(phase_stats(per, phases))
    out["resid"] = w2.resid()
    x = w2.solution()
    w2.F.close()
    return out, x


def secondary_2d(torch, local, args):
    """The 2D 1023^2 workload in FP64 beside the reference's CPU code on the
    full workload (one sample): a like-for-like GPU / CPU pair."""
    w = WORKLOADS["2d-1023"]
    from mfgpu import MFGPU_FP64
    work = SingleWork(w, 0, local, MFGPU_FP64)
    work.stream = torch.cuda.Stream()
    work.F.set_stream(work.stream.cuda_stream)
    work.to_device(torch)
    for _ in range(3):
        work.step()
    torch.cuda.synchronize()
    ms, per, phases = timed_steps(torch, work, args.steps)
    fl = work.step_flops()
    out = {"workload": f"2d-1023 ({w['label']})", "precision": "fp64",
           "fp64": dict({"steps": args.steps, "ms_per_step": ms / args.steps,
                         "value": fl * args.steps / (ms * 1e-3) / 1e12, "unit": "TFLOP/s",
                         "resid": work.resid()}, **phase_stats(per, phases))}
    work.F.close()
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        a1, a2, A1, A2, mod, b, _ = make_problem(w)
        res = reference_time(2, w["N"], w["max_side"], a1, a2, b, threads, reps=1)
        if res is not None:
            t = res["factor_s"][0] + res["update_s"][0] + res["solve_s"][0]
            out["reference_cpu"] = {
                "value": ref_step_flops(res, w["nrhs"]) / t / 1e12, "unit": "TFLOP/s",
                "ms_per_step": t * 1e3, "cores": threads, "kind": "reference",
                "sample": f"1 x (factor + update + {w['nrhs']}-RHS solve) of the full workload, "
                          f"OPENBLAS_NUM_THREADS={threads}"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="3d-127", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip timing the other precision for the mixed-vs-FP64 comparison")
    ap.add_argument("--compare-steps", type=int, default=5,
                    help="timed steps of the other precision (bounded: FP64 3d-127 is ~6.5 s/step)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the 2D 1023^2 FP64 line beside the reference's CPU code")
    ap.add_argument("--json-out", default=None)
    ap.add_argument("--autotune", type=int, default=0, metavar="REPS",
                    help="pick each level's kernel by timing (mfgpu_autotune, REPS runs per "
                         "candidate) during set-up, before the warm-up; 0 = size rules")
    ap.add_argument("--rate", type=float, default=4.0, help="serving: arrivals per second")
    ap.add_argument("--requests", type=int, default=24, help="serving: requests in the stream")
    ap.add_argument("--slots", type=int, default=8, help="serving: requests per batch")
    ap.add_argument("--serve-reference", action="store_true",
                    help="serving: also time the reference's CPU Update + Solve of the first "
                         "request on the host cores (minutes: it factors the base first)")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        if w.get("serve"):
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no serving loop; its Update + Solve per request "
                              "is timed by the 3d workloads"}))
            return 0
        return run_reference_arm(args, w)
    if w.get("serve"):
        return run_serve(args, w)

    import torch
    import torch.distributed as dist

    from mfgpu import MFGPU_FP64, MFGPU_MIXED

    prec = MFGPU_MIXED if args.precision == "mixed" else MFGPU_FP64
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    Work = BatchWork if w.get("batch") else SingleWork
    problem = None if w.get("batch") else make_problem(w, rank)
    work = Work(w, rank, local, prec, problem)
    F = work.F
    work.stream = torch.cuda.Stream()
    F.set_stream(work.stream.cuda_stream)
    work.to_device(torch)
    torch.cuda.synchronize()
    tuned = work.F.autotune(args.autotune) if args.autotune > 0 else None   # set-up, untimed
    warm = max(3, args.warmup)
    for _ in range(warm):
        work.step()
    torch.cuda.synchronize()
    resid = work.resid()      # correctness of what is timed, in FP64 on the host
    iters = F.stats()["iterations"] if args.precision == "mixed" else 0
    step_fl = work.step_flops()

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    F.profile(True)
    F.profile_reset()
    launches0 = F.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    ms_total, per, phases = timed_steps(torch, work, args.steps)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = F.kernel_launches() - launches0
    prof = F.profile_read()
    F.profile(False)
    value, ms_max, _ = whole_job(ms_total, args.steps * step_fl, "cuda")
    x_this = work.solution() if rank == 0 else None

    # end to end through the public API with pinned host buffers
    work.e2e_setup(torch)
    work.e2e_step()
    torch.cuda.synchronize()
    ee0 = torch.cuda.Event(enable_timing=True)
    ee1 = torch.cuda.Event(enable_timing=True)
    ee0.record(work.stream)
    for _ in range(args.steps):
        work.e2e_step()
    ee1.record(work.stream)
    ee1.synchronize()
    e2e_value, _, _ = whole_job(ee0.elapsed_time(ee1), args.steps * step_fl, "cuda")
    h2d, d2h = work.e2e_bytes()

    # roofline of the dominant kernel class in the timed region
    peaks, peak_src = measured_peaks()
    dom = max((k for k in prof if prof[k]["ms"] > 0), key=lambda k: prof[k]["ms"])
    roof = None
    if rank == 0:
        roof = roofline(torch, dom, prof[dom], peaks, peak_src, args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = work.cpu_baseline(os.cpu_count() or 1)

    config = work.config(args, args.precision)
    if tuned is not None:
        config["autotune"] = {"reps": args.autotune, "level_kernels_root_first": tuned}
    flops_bd = work.flops_breakdown()
    this = {"steps": args.steps, "warmup": warm, "ms_per_step": ms_max / args.steps,
            "value": value, "resid": resid}
    this.update(phase_stats(per, phases))
    work.F.close()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    # the metric compares mixed precision with FP64: the other precision on the
    # same workload and step, and the forward error between the two solutions
    comparison = None
    if not args.no_compare and world == 1:
        other = MFGPU_FP64 if prec == MFGPU_MIXED else MFGPU_MIXED
        that, x_that = other_precision_run(torch, w, rank, local, other, args, problem)
        mixed_, fp64_ = (this, that) if prec == MFGPU_MIXED else (that, this)
        x_mixed, x_fp64 = (x_this, x_that) if prec == MFGPU_MIXED else (x_that, x_this)
        comparison = {"fp64": fp64_, "mixed": mixed_,
                      "mixed_speedup": fp64_["ms_per_step"] / mixed_["ms_per_step"],
                      "forward_error_mixed_vs_fp64": forward_error(x_mixed, x_fp64),
                      "note": "same workload and step; device time (CUDA events); residuals of "
                              "the updated system in FP64 on the host; the FP64 path is checked "
                              "against the reference (oracle) in the GPU tests"}
        torch.cuda.empty_cache()

    secondary = None
    if (rank == 0 and world == 1 and not args.no_secondary and args.workload == "3d-127"):
        secondary = secondary_2d(torch, local, args)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": warm, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": dtype_of(args.precision),
            "data": "synthetic (seeded coefficients and right-hand sides)",
            "config": config,
            "step_s_p50": this["step_ms_p50"] * 1e-3, "step_s_p99": this["step_ms_p99"] * 1e-3,
            "update_solve_s_p50": this["update_solve_ms_p50"] * 1e-3,
            "update_solve_s_p99": this["update_solve_ms_p99"] * 1e-3,
            "resid": resid,
            "refine_iterations": iters,
            "flops_per_step": flops_bd,
            "phases_ms_p50": {k: this[k] for k in ("factor_ms_p50", "update_ms_p50",
                                                   "solve_ms_p50")},
            "kernel_classes": {k: {"launches": v["launches"], "ms": v["ms"]} for k, v in prof.items()},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "TFLOP/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "precision_comparison": comparison,
        }
        if secondary is not None:
            line["secondary_2d1023_fp64"] = secondary
        s = json.dumps(line)
        print(s)
        if args.json_out:
            with open(args.json_out, "w") as f:
                f.write(s + "\n")
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# profiling class -> the kernel it times
KERNEL_OF = {"front": "k_front_small", "coop": "k_level_coop", "tc": "k_trail_tc",
             "assemble": "k_tasks", "solve": "k_solve_*", "apply": "k_apply_*",
             "potrf": "k_potrf", "trsm": "k_trsm", "syrk": "k_syrk"}


def roofline(torch, dom, P, peaks, peak_src, args):
    kern = KERNEL_OF.get(dom, dom)
    common = {"kernel": kern, "class": dom, "launches": P["launches"],
              "avg_launch_ms": P["ms"] / max(1, P["launches"]),
              "traffic": traffic_for(kern, args.workload, args.precision)}
    ach = P["flops"] / (P["ms"] * 1e-3) / 1e12
    if dom == "tc":
        split = {"1": 1, "tf32": 1, "bf16": 1}.get(os.environ.get("MFGPU_TC_SPLIT", "3"), 3)
        pk = float(peaks["bf16_tflops"]) / 2.0
        return dict(common, bound="tensor", achieved=ach, peak=pk, unit="TFLOP/s", frac=ach / pk,
                    achieved_executed=ach * split,
                    peak_source=f"{peak_src} bf16_tflops / 2 (MEASURED_PEAKS.json, else the "
                                "pool's fallback): the dense TF32 rate is half the BF16 rate; "
                                "achieved counts the algorithmic flops once, the kernel executes "
                                f"{split} TF32 products per flop")
    if dom in ("potrf", "trsm", "syrk", "front", "coop"):
        dt, nm = (torch.float32, "SGEMM (float32") if args.precision == "mixed" else \
            (torch.float64, "DGEMM (float64")
        pk = measured_gemm_peak(torch, dt)
        return dict(common, bound="tensor", achieved=ach, peak=pk, unit="TFLOP/s", frac=ach / pk,
                    peak_source=f"measured cuBLAS {nm} matmul 8192^3, TF32 off) on this GPU; "
                                "the factor's precision has no entry in MEASURED_PEAKS.json")
    ach = P["bytes"] / (P["ms"] * 1e-3) / 1e9
    pk = float(peaks["hbm_gbs"])
    return dict(common, bound="hbm", achieved=ach, peak=pk, unit="GB/s", frac=ach / pk,
                peak_source=f"{peak_src} hbm_gbs (MEASURED_PEAKS.json)")


def traffic_for(kernel, workload, precision):
    """DRAM bytes (read + write) per launch of `kernel` in this workload, from
    the ncu capture summarised in profiles/traffic.json, when one exists."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.isfile(p):
        with open(p) as f:
            d = json.load(f)
        v = d.get(f"{kernel}/{workload}/{precision}")
        if isinstance(v, dict):
            return v.get("dram_bytes_per_launch")
    return None


def run_serve(args, w):
    """Update serving (3D 95^3 base, the serving configuration): a stream of requests with
    Poisson arrivals against a resident factorization; each request changes
    the coefficients of one box and brings right-hand sides.  Reports
    throughput and p50/p99 latency (wall clock from submission to the result
    on the host, queueing included) and the algorithmic TFLOP/s of the
    completed requests (their root-path refactorizations and solves)."""
    import threading
    import torch
    from mfgpu import MF2D, MF3D, MFGPU_FP64, MFGPU_MIXED, Server, Symbolic
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    prec = MFGPU_MIXED if args.precision == "mixed" else MFGPU_FP64
    N = w["N"]
    seed = w["seed"] + 1000 * rank
    a = stencil.loguniform_coefficients(N, w["lo"], w["hi"], seed)
    A = stencil.build_laplacian(a)
    F = (MF3D(A, N[0], N[1], N[2], 1, w["max_side"], device=local, precision=prec)
         if w["dim"] == 3 else MF2D(A, N[0], N[1], 1, w["max_side"], device=local, precision=prec))
    F.Factor()
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    reqs = []
    for _ in range(args.requests):
        side = int(rng.integers(w["side"][0], w["side"][1] + 1))
        lo = [int(rng.integers(0, n - side + 1)) for n in N]
        factor = float(w["lo"] * (w["hi"] / w["lo"]) ** rng.random())
        k = int(rng.integers(w["nrhs"][0], w["nrhs"][1] + 1))
        b = rng.uniform(-1, 1, size=(A.n, k))
        reqs.append((lo, [l + side for l in lo], factor, b))
    gaps = rng.exponential(1.0 / args.rate, size=args.requests)
    S = Symbolic(w["dim"], N, 1, w["max_side"])
    fronts = [S.front(f) for f in range(S.n_fronts)]
    solve_unit = sum(2.0 * (f["n"] ** 2 + 2.0 * f["n"] * f["m"]) for f in fronts)
    free_gb = torch.cuda.mem_get_info()[0] / 2 ** 30
    # per batch member: values, coefficients, block inverses; the view's workspaces
    slot_gb = 0.25 * (1 if prec == MFGPU_MIXED else 2)
    pool_gb = max(4.0, free_gb - 8.0 - args.slots * slot_gb)
    srv = Server(F, a, slots=args.slots, pool_gb=pool_gb)
    # one warm-up request outside the measurement
    srv.wait(srv.submit(reqs[0][0], reqs[0][1], reqs[0][2], reqs[0][3][:, :1]))
    results = [None] * len(reqs)
    tickets = [None] * len(reqs)
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()

    def producer():
        t = t0
        for i, (lo, hi, f, b) in enumerate(reqs):
            t += gaps[i]
            d = t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets[i] = srv.submit(lo, hi, f, b)

    th = threading.Thread(target=producer)
    th.start()
    for i in range(len(reqs)):
        while tickets[i] is None:
            time.sleep(0.0005)
        results[i] = srv.wait(tickets[i])
    th.join()
    makespan = time.perf_counter() - t0
    clk = clocks.stop()
    lat = [r[1]["latency_seconds"] for r in results]
    work = 0.0
    for (lo, hi, f, b), (x, info) in zip(reqs, results):
        dirty, fl = S.dirty([i + j * N[0] + k * N[0] * N[1]
                             for k in range(max(0, lo[2] - 1), min(N[2], hi[2] + 1))
                             for j in range(max(0, lo[1] - 1), min(N[1], hi[1] + 1))
                             for i in range(max(0, lo[0] - 1), min(N[0], hi[0] + 1))])
        work += fl + solve_unit * b.shape[1]
    # correctness of what was timed: FP64 residual of one request's answer
    lo, hi, f, b = reqs[-1]
    Ar = stencil.build_laplacian(stencil.scale_box(a, lo, hi[0] - lo[0], f))
    x = results[-1][0]
    resid = max(float(np.linalg.norm(Ar.matvec(x[:, c]) - b[:, c]) / np.linalg.norm(b[:, c]))
                for c in range(b.shape[1]))
    srv.close()
    line = {
        "metric": "update-serving throughput (algorithmic TFLOP/s of completed requests) and "
                  "latency p50/p99",
        "value": work / makespan / 1e12, "unit": "TFLOP/s", "n_gpus": 1, "steps": len(reqs),
        "warmup": 1, "ms_per_step": makespan / len(reqs) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(args.precision),
        "data": "synthetic (seeded coefficients, boxes, factors and right-hand sides)",
        "config": {"workload": f"{args.workload} (3D {N[0]}^3 7-point, a log-U[{w['lo']},{w['hi']}], "
                               f"maxSideLength {w['max_side']}; {len(reqs)} requests, Poisson "
                               f"arrivals at {args.rate}/s, box side {w['side'][0]}-{w['side'][1]}, "
                               f"{w['nrhs'][0]}-{w['nrhs'][1]} RHS)",
                   "batch_capacity": args.slots, "pool_gb": round(pool_gb, 1),
                   "precision": args.precision,
                   "timing": "wall clock, submission to result on the host"},
        "requests_per_s": len(reqs) / makespan,
        "latency_s": {"p50": statistics.median(lat), "p99": pct(lat, 99), "max": max(lat)},
        "queued_s_p50": statistics.median(r[1]["queued_seconds"] for r in results),
        "fronts_per_request_p50": statistics.median(r[1]["fronts"] for r in results),
        "batch_size": {"p50": statistics.median(r[1]["batch"] for r in results),
                       "max": max(r[1]["batch"] for r in results)},
        "resid": resid, "clocks": clk,
        "e2e": {"value": work / makespan / 1e12, "unit": "TFLOP/s",
                "h2d_bytes_per_step": int(np.mean([b.nbytes for *_, b in reqs])),
                "d2h_bytes_per_step": int(np.mean([b.nbytes for *_, b in reqs]))},
    }
    F.close()
    if args.serve_reference:
        # the reference serves a request as Update + Solve on its own factored
        # base (no batching, no serving loop); time the first request
        lo, hi, f, b = reqs[0]
        threads = os.cpu_count() or 1
        res = reference_time(w["dim"], N, w["max_side"], a,
                             stencil.scale_box(a, lo, hi[0] - lo[0], f),
                             np.ascontiguousarray(b.T), threads, reps=1)
        if res is not None:
            line["reference_cpu"] = {
                "update_s": res["update_s"][0], "solve_s": res["solve_s"][0],
                "update_solve_s": res["update_s"][0] + res["solve_s"][0],
                "base_factor_s": res["factor_s"][0], "cores": threads, "kind": "reference",
                "sample": f"request 0 (box side {hi[0] - lo[0]}, factor {f:.3g}, "
                          f"{b.shape[1]} RHS) as the reference's Update + Solve on its factored "
                          f"base, OPENBLAS_NUM_THREADS={threads}"}
    print(json.dumps(line))
    if args.json_out:
        with open(args.json_out, "w") as fo:
            fo.write(json.dumps(line) + "\n")
    return 0


if __name__ == "__main__":
    sys.path.insert(0, PKG)
    sys.exit(main())
