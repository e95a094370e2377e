#!/usr/bin/env python
"""Benchmark of the approxchol_lap solve phase on B200.

Workload: the 100x100x100 3D grid (1,000,000 vertices, 6-neighbour) with
edge weights log-uniform in [1e-3, 1] (seeded); each solve has one zero-mean
Gaussian right-hand side; one step solves --rhs (default 64) independent
right-hand sides in one batched launch; tol 1e-8 on the true relative
residual |L x - b| / |b|, FP32 PCG (SpMV and LDLinv sweeps) inside FP64
iterative refinement.  The factor is built once on the host with the
reference's :deg elimination (not timed; its time is reported as factor_s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl acgpu|reference]

Metric: solves/s (whole job; replicas: each GPU solves its own right-hand
sides on its own copy of the factor, no collective on the data path).
`value` times device-resident inputs; `e2e` goes through the C ABI entry
acg_solve with pinned host buffers, host<->device copies inside the timed
region.  --impl reference times the CPU restatement of the reference's
solve (pcg + LDLsolver, single-threaded per solve) on all host cores.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for _p in (ROOT / "laplacians.jl_b200", ROOT / "oracle"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "solves/s at |Lx-b|/|b|<=1e-8 (mixed FP32/FP64 PCG, 1M-vertex weighted 3D grid)"
GRID_SIDE = 100
WEIGHT_SEED = 7
FACTOR_SEED = 1
TOL = 1e-8
MAXITS = 2000


def build_workload():
    from acgpu import generators as G
    import acgpu
    a = G.grid3(GRID_SIDE, weights="loguniform", seed=WEIGHT_SEED)
    acgpu.seed(FACTOR_SEED)
    t = time.perf_counter()
    ldli = acgpu.approx_chol(a)
    return a, ldli, time.perf_counter() - t


def rhs(n, seed):
    b = np.random.default_rng(seed).standard_normal(n)
    return b - b.mean()


def config(n, extra=None):
    c = {"workload": f"grid3({GRID_SIDE}) log-uniform weights [1e-3,1], 1 zero-mean Gaussian RHS per solve, tol 1e-8",
         "n": n, "precision": "fp32 PCG in fp64 refinement",
         "l2": "inputs larger than L2 (factor + Laplacian > 126 MB), no flush"}
    if extra:
        c.update(extra)
    return c


# ---- clocks ---------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.file:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---- CPU baseline (the oracle port) ------------------------------------------

def cpu_solve_time(a, ldli, b, its_hint, budget_s=25.0):
    """One-thread time of one solve of the workload with the CPU restatement.
    Runs the full solve when it fits the budget; otherwise times a bounded
    number of PCG iterations and scales to its_hint iterations."""
    import oracle as O
    orc = O.OracleSolver(a, ldli)
    t = time.perf_counter()
    orc(b, tol=TOL, maxits=2)
    t2 = time.perf_counter() - t
    per_it = t2 / 3.0  # the initial preconditioner application + 2 iterations
    full = per_it * (its_hint + 1)
    if full <= budget_s:
        t = time.perf_counter()
        _, its, _, _ = orc(b, tol=TOL, maxits=MAXITS)
        return time.perf_counter() - t, f"one full solve at tol 1e-8 ({its} PCG iterations, FP64)"
    m = max(2, int(budget_s / per_it) - 1)
    t = time.perf_counter()
    orc(b, tol=0.0, maxits=m)
    el = time.perf_counter() - t
    return el / (m + 1) * (its_hint + 1), f"{m} FP64 PCG iterations timed, scaled to {its_hint} iterations"


# ---- arms -------------------------------------------------------------------------

def dist_setup(gpus):
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    return rank, world, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_acgpu(args):
    import torch
    import acgpu
    from acgpu._lib import AcgSolveInfo, check, lib

    rank, world, local = dist_setup(args.gpus)
    a, ldli, factor_s = build_workload()
    n = a.shape[0]
    t = time.perf_counter()
    dev = acgpu.DeviceLapSolver(a, ldli)
    upload_s = time.perf_counter() - t
    L = lib()
    prec = 1 if args.precision == "mixed" else 0
    k = args.rhs

    # device-resident right-hand sides: k independent columns per step, distinct per rank
    nsteps = args.warmup + args.steps
    B = torch.empty((nsteps, k, n), dtype=torch.float64, device="cuda")
    for i in range(nsteps):
        for c in range(k):
            B[i, c] = torch.from_numpy(rhs(n, 1_000_000 * rank + 1000 * i + c))
    X = torch.empty((k, n), dtype=torch.float64, device="cuda")
    infos = (AcgSolveInfo * k)()

    def solve_step(i):
        if k == 1:
            rc = L.acg_solve_device(dev._h, ctypes.c_void_p(B[i].data_ptr()), ctypes.c_void_p(X.data_ptr()), TOL,
                                    MAXITS, float("inf"), 5, prec, infos)
        else:
            rc = L.acg_solve_batch_device(dev._h, ctypes.c_void_p(B[i].data_ptr()), ctypes.c_void_p(X.data_ptr()),
                                          k, n, TOL, MAXITS, float("inf"), 5, prec, infos)
        check(rc)
        return [(infos[c].iterations, infos[c].refinements, infos[c].true_relres, infos[c].status) for c in range(k)]

    for i in range(args.warmup):
        solve_step(i)
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    results = []
    with ClockSampler(local) as clk:
        time.sleep(0.5)  # let the sampler start before the timed region
        torch.cuda.synchronize()
        e0.record()
        for i in range(args.warmup, nsteps):
            results += solve_step(i)
        e1.record()
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    clocks = clk.summary()
    bad = [r for r in results if r[3] != 0 or r[2] > TOL]
    if bad:
        raise RuntimeError(f"{len(bad)} solves missed the tolerance: {bad[:3]}")
    its = np.array([r[0] for r in results], dtype=float)
    refs = np.array([r[1] for r in results], dtype=float)
    res = np.array([r[2] for r in results])

    # end to end: pinned host blocks through acg_solve (H2D + D2H inside the timed region)
    hb = torch.empty((args.steps, k, n), dtype=torch.float64, pin_memory=True)
    hx = torch.empty((k, n), dtype=torch.float64, pin_memory=True)
    hb_np = hb.numpy()
    hx_np = hx.numpy()
    for i in range(args.steps):
        for c in range(k):
            hb_np[i, c] = rhs(n, 5_000_000 + 1_000_000 * rank + 1000 * i + c)
    hb_flat = [np.ascontiguousarray(hb_np[i]).reshape(-1) for i in range(args.steps)]
    hx_flat = hx_np.reshape(-1)
    check(L.acg_solve(dev._h, hb_flat[0], hx_flat, k, n, TOL, MAXITS, float("inf"), 5, prec, infos))
    barrier(world)
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record()
    for i in range(args.steps):
        check(L.acg_solve(dev._h, hb_flat[i], hx_flat, k, n, TOL, MAXITS, float("inf"), 5, prec, infos))
    e3.record()
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(e2.elapsed_time(e3), world)

    # one right-hand side alone: latency of a single solve
    single = []
    for i in range(3):
        t0 = time.perf_counter()
        check(L.acg_solve_device(dev._h, ctypes.c_void_p(B[i, 0].data_ptr()), ctypes.c_void_p(X.data_ptr()), TOL,
                                 MAXITS, float("inf"), 5, prec, infos))
        single.append(infos[0].solve_ms)

    # roofline of the dominant kernel (the forward LDLinv sweep), timed live
    kt = dev.time_kernels_batch(k, args.precision, reps=5) if k > 1 else dev.time_kernels(args.precision, reps=5)
    stats = dev.stats()
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    achieved = kt["forward_bytes"] / (kt["forward_ms"] * 1e-3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / ("kb_sweep_forward_grid3_100_k64.md" if k > 1 else "k_sweep_forward_grid3_100.md")
    if prof.exists() and GRID_SIDE == 100:
        import re
        m = re.search(r"dram_bytes_per_launch:\s*(\d+)", prof.read_text())
        traffic = int(m.group(1)) if m else None

    # our kernel launches per step: set-up/wrap-up 3, per refinement 8, per inner iteration 8 (9 for k = 1)
    per_it = kt["launches_per_iteration"] if k == 1 else 8
    launches = args.steps * (3 + refs.max() * 8 + its.max() * per_it)

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            t_cpu, sample = cpu_solve_time(a, ldli, rhs(n, 424242), int(round(its.mean())))
            cpu = {"value": 1.0 / t_cpu, "unit": "solves/s", "cores": 1, "kind": "port", "sample": sample}
        value = world * args.steps * k / (ms * 1e-3)
        kern = (f"kb_sweep<float,{k // 8 if k >= 8 else 1},forward> (batched LDLinv forward sweep, {k} columns)"
                if k > 1 else "k_sweep<float,forward> (LDLinv forward sweep)")
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (SpMV, sweeps) / f64 (residual, dots, correction)"
            if prec == 1 else "f64", "data": "synthetic (seeded grid weights and Gaussian RHS)",
            "config": config(n, {"parallelism": f"replicas x{world}", "rhs_per_step": k,
                                 "batching": f"{k} independent single-RHS solves per step in one batched launch",
                                 "pcg_iterations_mean": float(its.mean()), "refinements_mean": float(refs.mean()),
                                 "true_relres_max": float(res.max()), "factor_s": factor_s, "upload_s": upload_s,
                                 "levels": stats["levels"], "factor_nnz": stats["nnz_factor"]}),
            "single_rhs": {"latency_ms": float(np.median(single)), "solves_per_s": 1e3 / float(np.median(single))},
            "e2e": {"value": world * args.steps * k / (e2e_ms * 1e-3), "unit": "solves/s",
                    "h2d_bytes_per_step": 8 * n * k, "d2h_bytes_per_step": 8 * n * k},
            "roofline": {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                         "algorithmic_bytes_per_launch": kt["forward_bytes"], "launch_ms": kt["forward_ms"],
                         "backward_ms": kt["backward_ms"], "spmv_ms": kt["spmv_ms"],
                         "spmv_gbs": kt["spmv_bytes"] / (kt["spmv_ms"] * 1e-3) / 1e9},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": int(round(launches)),
        }
        print(json.dumps(line), flush=True)
    dev.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference(args):
    """The reference's solve on the host cores: the CPU restatement of pcg +
    LDLsolver (oracle port), one independent solve per thread."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import oracle as O
    a, ldli, factor_s = build_workload()
    n = a.shape[0]
    threads = max(1, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count())
    solver = O.OracleSolver(a, ldli)  # read-only; the C solve keeps its state on the stack/heap per call
    budget = 150.0

    def step(seed_base):
        res = [None] * threads

        def work(k):
            x, its, rc, nr = solver(rhs(n, seed_base + k), tol=TOL, maxits=MAXITS)
            res[k] = (its, rc)

        ths = [threading.Thread(target=work, args=(k,)) for k in range(threads)]
        t = time.perf_counter()
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        return time.perf_counter() - t, res

    t_first, res = step(0)  # warm-up (also sizes the sample)
    steps = max(1, min(args.steps, int(budget / max(t_first, 1e-3))))
    warm = min(args.warmup - 1, int(30.0 / max(t_first, 1e-3)))
    for w in range(max(0, warm)):
        step(100 + w * threads)
    total = 0.0
    its = []
    for s in range(steps):
        el, res = step(10000 + s * threads)
        total += el
        its += [r[0] for r in res]
    value = steps * threads / total
    sample = (f"{steps} step(s) of {threads} concurrent full solves (one per host thread), tol 1e-8, FP64 CPU "
              f"restatement of pcg + LDLsolver; mean {np.mean(its):.1f} PCG iterations")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(n, {"parallelism": f"{threads} host threads", "factor_s": factor_s}),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="acgpu", choices=["acgpu", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--side", type=int, default=GRID_SIDE, help="grid side (100 = the benchmark workload)")
    ap.add_argument("--rhs", type=int, default=64, help="independent right-hand sides per step (batched)")
    args = ap.parse_args()
    globals()["GRID_SIDE"] = args.side
    if args.warmup < 3 and args.impl == "acgpu":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_acgpu(args)


if __name__ == "__main__":
    main()
