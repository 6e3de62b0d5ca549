#!/usr/bin/env python3
"""Benchmark: factor + localized update + solve on one B200 per rank.

Workload (default): 2D 5-point variable-coefficient Laplacian on a 1023 x 1023
interior grid (n = 1,046,529), node coefficients iid log-uniform in [0.1, 10]
from a fixed seed, leaf parameter 8 (leaf boxes of 15 x 15 cells, 16 x 16
cells per leaf period), 4 right-hand sides iid uniform[-1, 1].  One step is
  1. a full factorization of the matrix (values resident in HBM),
  2. a localized update: coefficients x10 on a 9 x 9-cell patch at a seeded
     position, refactoring only the root paths of the leaves it touches,
  3. a 4-RHS solve with the updated factorization.
The metric is algorithmic TFLOP/s of that step: Cholesky-form flops
sum(n^3/3 + n^2 m + n m^2) over the factored fronts, the same over the fronts
the update refactors, and 2(n^2 + 2nm) per front and right-hand side for the
solve, divided by the device time of the step.  The same flop count is used for
the reference arm, whose LU-based code performs about 2.4x more arithmetic.

Multi-GPU: the path does not shard (one problem per GPU); N ranks run N
independent replicas ("weak" scaling) and `value` is the aggregate.

`--impl reference` times the reference's own CPU implementation
(oracle/_ref/ref_harness, compiled from the reference sources) on the host
cores with every host thread.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "updating-multifrontal_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

from mfgpu import stencil  # noqa: E402

SEED0 = 20261203
WORKLOADS = {
    # the 2D variable-coefficient workload with 4 right-hand sides
    "2d-1023": dict(dim=2, N=(1023, 1023), max_side=8, lo=0.1, hi=10.0, nrhs=4, patch=9,
                    factor=10.0, seed=SEED0 + 2),
    # the CPU-runnable 2D workload (a = 1, leaf parameter 4, one RHS)
    "2d-127": dict(dim=2, N=(127, 127), max_side=4, lo=1.0, hi=1.0, nrhs=1, patch=9,
                   factor=10.0, seed=SEED0 + 1),
    # the 3D workload (log-uniform [0.1, 100], leaf parameter 4, one RHS)
    "3d-127": dict(dim=3, N=(127, 127, 127), max_side=4, lo=0.1, hi=100.0, nrhs=1, patch=9,
                   factor=10.0, seed=SEED0 + 3),
    # a smaller 3D case of the same kind (profiling captures, quick checks)
    "3d-63": dict(dim=3, N=(63, 63, 63), max_side=4, lo=0.1, hi=100.0, nrhs=1, patch=5,
                  factor=10.0, seed=SEED0 + 4),
}


def make_problem(w, rank=0):
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
    return a1, a2, A1, A2, mod, b


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


def reference_time(w, a1, a2, b, threads, reps=1, solve_reps=1, timeout=3000):
    """Run the compiled reference (oracle/_ref) in timing mode; returns its JSON."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refio
    if not refio.have_reference():
        return None
    with tempfile.TemporaryDirectory() as d:
        return refio.time_reference(d, w["dim"], w["N"], 1, w["max_side"], a1, a2, b,
                                    reps=reps, solve_reps=solve_reps, threads=threads,
                                    timeout=timeout)


def front_sizes(w):
    from mfgpu import Symbolic
    S = Symbolic(w["dim"], w["N"], 1, w["max_side"])
    return [(S.front(f)["n"], S.front(f)["m"]) for f in range(S.n_fronts)]


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
    return model, os.cpu_count() or 1


def run_reference_arm(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    a1, a2, A1, A2, mod, b = make_problem(w)
    fl = front_sizes(w)
    factor_fl = sum(n ** 3 / 3.0 + n * n * m + n * m * m for n, m in fl)
    threads = os.cpu_count() or 1
    # one warm-up sample, then `steps` samples; each sample = factor + update +
    # nrhs solves of the full workload, bounded to a few minutes in total
    upd_fl = update_flops(w, mod)
    sfl = solve_flops(fl, w["nrhs"])
    res = reference_time(w, a1, a2, b, threads, reps=1 + max(1, args.steps), solve_reps=1)
    model, ncpu = cpu_info()
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference harness oracle/_ref/ref_harness not built"}))
        return 0
    tf, tu, ts = res["factor_s"][1:], res["update_s"][1:], res["solve_s"][1:]
    steps = [tf[i] + tu[i] + ts[i] for i in range(len(tf))]
    step_fl = factor_fl + upd_fl + sfl
    t = statistics.median(steps)
    value = step_fl / t / 1e12
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s",
        "n_gpus": args.gpus, "steps": len(steps), "warmup": 1, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 factor + f64 refinement",
        "data": "synthetic (seeded coefficients and right-hand sides)",
        "config": config_of(w, args),
        "phases_s": {"factor_p50": statistics.median(tf), "update_p50": statistics.median(tu),
                     "solve_p50": statistics.median(ts), "step_p99": float(np.percentile(steps, 99))},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(steps)} x (factor + update + {w['nrhs']}-RHS solve) of "
                                   f"the full workload, OPENBLAS_NUM_THREADS={threads}",
                         "cpu": model},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def update_flops(w, mod):
    """Flops of the fronts a localized update refactors (root paths of dirty leaves)."""
    from mfgpu import Symbolic
    S = Symbolic(w["dim"], w["N"], 1, w["max_side"])
    return S.dirty(mod)[1]


METRIC = "factor+update+solve TFLOP/s (Cholesky-form algorithmic flops), FP64 on 1 B200"


def config_of(w, args):
    return {"workload": args.workload + (" (2D 1023x1023 5-point, a log-U[0.1,10], leaf 15x15, "
                                         "4 RHS, 9x9 patch x10 update)" if args.workload == "2d-1023"
                                         else ""),
            "grid": list(w["N"]), "max_side_length": w["max_side"], "nrhs": w["nrhs"],
            "precision": args.precision, "parallelism": f"replicas x{args.gpus}",
            "l2": "inputs larger than L2 (front arena > 126 MB)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="2d-1023", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--json-out", default=None)
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args, w)

    import torch
    import torch.distributed as dist

    from mfgpu import MF2D, MF3D, MFGPU_FP64, MFGPU_MIXED

    prec = MFGPU_MIXED if args.precision == "mixed" else MFGPU_FP64
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    a1, a2, A1, A2, mod, b = make_problem(w, rank)
    n, nnz, nrhs = A1.n, A1.nnz, w["nrhs"]
    if w["dim"] == 2:
        F = MF2D(A1, w["N"][0], w["N"][1], 1, w["max_side"], device=local, precision=prec)
    else:
        F = MF3D(A1, w["N"][0], w["N"][1], w["N"][2], 1, w["max_side"], device=local,
                 precision=prec)
    stream = torch.cuda.Stream()
    F.set_stream(stream.cuda_stream)
    dv1 = torch.from_numpy(A1.val).to("cuda")
    dv2 = torch.from_numpy(A2.val).to("cuda")
    db = torch.from_numpy(np.ascontiguousarray(b)).to("cuda")      # (nrhs, n): column-major n x nrhs
    dx = torch.empty_like(db)
    torch.cuda.synchronize()

    def step():
        F.refactor_device(dv1.data_ptr(), nnz)
        F.update_device(dv2.data_ptr(), nnz, mod)
        F.solve_device(db.data_ptr(), dx.data_ptr(), nrhs, n)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    # correctness of what is timed: residual of the updated system in FP64
    x = dx.cpu().numpy()
    resid = max(float(np.linalg.norm(A2.matvec(x[r]) - b[r]) / np.linalg.norm(b[r]))
                for r in range(nrhs))
    info = F.info()
    fl = front_sizes(w)
    upd_fl = update_flops(w, mod)
    step_fl = info["factor_flops"] + upd_fl + solve_flops(fl, nrhs)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    F.profile(True)
    F.profile_reset()
    launches0 = F.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    with torch.cuda.stream(stream):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        per_step = []
        for _ in range(args.steps):
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            step()
            s1.record(stream)
            per_step.append((s0, s1))
        e1.record(stream)
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = F.kernel_launches() - launches0
    prof = F.profile_read()
    F.profile(False)
    ms_total = e0.elapsed_time(e1)
    step_ms = [a.elapsed_time(c) for a, c in per_step]
    t = torch.tensor([ms_total], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps * step_fl / (ms_max * 1e-3) / 1e12

    # end to end through the public API with pinned host buffers
    hv1 = torch.from_numpy(A1.val).pin_memory()
    hv2 = torch.from_numpy(A2.val).pin_memory()
    hb = torch.from_numpy(np.ascontiguousarray(b)).pin_memory()
    hx = torch.empty_like(hb).pin_memory()
    mod32 = np.ascontiguousarray(mod, np.int32)
    F.set_stream(stream.cuda_stream)

    def e2e_step():
        F.refactor_host_ptr(hv1.data_ptr(), nnz)
        F.update_host_ptr(hv2.data_ptr(), nnz, mod32)
        F.solve_host_ptr(hb.data_ptr(), hx.data_ptr(), nrhs, n)

    e2e_step()
    torch.cuda.synchronize()
    ee0 = torch.cuda.Event(enable_timing=True)
    ee1 = torch.cuda.Event(enable_timing=True)
    ee0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    ee1.record(stream)
    ee1.synchronize()
    e2e_ms = ee0.elapsed_time(ee1)
    te = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps * step_fl / (float(te.item()) * 1e-3) / 1e12
    h2d = 2 * nnz * 8 + n * nrhs * 8 + mod32.size * 4
    d2h = n * nrhs * 8

    # roofline of the dominant kernel class in the timed region
    peaks, peak_src = measured_peaks()
    dom = max((k for k in prof if prof[k]["ms"] > 0), key=lambda k: prof[k]["ms"])
    P = prof[dom]
    roof = None
    if rank == 0:
        kern = KERNEL_OF.get(dom, dom)
        common = {"kernel": kern, "class": dom, "launches": P["launches"],
                  "avg_launch_ms": P["ms"] / max(1, P["launches"]),
                  "traffic": traffic_for(kern, args.workload, args.precision)}
        ach = P["flops"] / (P["ms"] * 1e-3) / 1e12
        if dom == "tc":
            split = int(os.environ.get("MFGPU_TC_SPLIT", "3"))
            pk = float(peaks["bf16_tflops"]) / 2.0
            roof = dict(common, bound="tensor", achieved=ach, peak=pk, unit="TFLOP/s", frac=ach / pk,
                        achieved_executed=ach * split,
                        peak_source=f"{peak_src} bf16_tflops / 2 (MEASURED_PEAKS.json): the dense "
                                    "TF32 rate is half the BF16 rate; achieved counts the "
                                    f"algorithmic flops once, the kernel executes {split} TF32 "
                                    "products per flop")
        elif dom in ("potrf", "trsm", "syrk", "front", "coop"):
            dt, nm = (torch.float32, "SGEMM (float32") if args.precision == "mixed" else \
                (torch.float64, "DGEMM (float64")
            pk = measured_gemm_peak(torch, dt)
            roof = dict(common, bound="tensor", achieved=ach, peak=pk, unit="TFLOP/s", frac=ach / pk,
                        peak_source=f"measured cuBLAS {nm} matmul 8192^3, TF32 off) on this GPU; "
                                    "the factor's precision has no entry in MEASURED_PEAKS.json")
        else:
            ach = P["bytes"] / (P["ms"] * 1e-3) / 1e9
            pk = float(peaks["hbm_gbs"])
            roof = dict(common, bound="hbm", achieved=ach, peak=pk, unit="GB/s", frac=ach / pk,
                        peak_source=f"{peak_src} hbm_gbs (MEASURED_PEAKS.json)")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        res = reference_time(w, a1, a2, b, threads, reps=1, solve_reps=1)
        if res is not None:
            tcpu = res["factor_s"][0] + res["update_s"][0] + res["solve_s"][0]
            model, _ = cpu_info()
            cpu = {"value": step_fl / tcpu / 1e12, "unit": "TFLOP/s", "cores": threads,
                   "kind": "reference",
                   "sample": f"1 x (factor + update + {nrhs}-RHS solve) of the full workload "
                             f"({tcpu:.2f} s), OPENBLAS_NUM_THREADS={threads}", "cpu": model}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 factor + f64 refinement",
            "data": "synthetic (seeded coefficients and right-hand sides)",
            "config": config_of(w, args),
            "step_ms_p50": statistics.median(step_ms),
            "step_ms_p99": float(np.percentile(step_ms, 99)),
            "resid": resid,
            "refine_iterations": F.stats()["iterations"] if args.precision == "mixed" else 0,
            "flops_per_step": {"factor": info["factor_flops"], "update": upd_fl,
                               "solve": solve_flops(fl, nrhs)},
            "kernel_classes": {k: {"launches": v["launches"], "ms": v["ms"]} for k, v in prof.items()},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "TFLOP/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
        }
        s = json.dumps(line)
        print(s)
        if args.json_out:
            with open(args.json_out, "w") as f:
                f.write(s + "\n")
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    F.close()
    return 0


# profiling class -> the kernel it times
KERNEL_OF = {"front": "k_front_small", "coop": "k_level_coop", "tc": "k_trail_tc",
             "assemble": "k_tasks", "solve": "k_solve_*", "apply": "k_apply_*",
             "potrf": "k_potrf", "trsm": "k_trsm", "syrk": "k_syrk"}


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


if __name__ == "__main__":
    sys.exit(main())
