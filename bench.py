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
`value` times device-resident inputs; `e2e` goes through the C ABI entries
acg_solve_async / acg_wait with pinned host buffers, every step's
host<->device copies inside the timed region (two steps in flight: one step's
copies overlap the previous step's solve).  --impl reference times the CPU restatement of the reference's
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


def build_workload_host_only():
    """The same graph and factor without the GPU library: the generators
    module is loaded by path (plain numpy/scipy, not through the acgpu package,
    whose import maps libacgpu.so) and the host elimination comes from
    libacghost.so, the CUDA-free host part of the product (the elimination
    stays on the host in both arms and is not timed)."""
    import importlib.util
    import types
    spec = importlib.util.spec_from_file_location(
        "acg_generators", ROOT / "laplacians.jl_b200" / "acgpu" / "generators.py")
    G = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(G)
    a = G.grid3(GRID_SIDE, weights="loguniform", seed=WEIGHT_SEED)
    L = ctypes.CDLL(str(ROOT / "laplacians.jl_b200" / "acgpu" / "libacghost.so"))
    L.acg_last_error.restype = ctypes.c_char_p
    state = np.zeros(4, dtype=np.uint64)
    ptr = lambda arr: arr.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    if L.acg_rng_seed(ctypes.c_uint64(FACTOR_SEED), ptr(state)) != 0:
        raise RuntimeError(L.acg_last_error().decode())
    n = a.shape[0]
    cp = a.indptr.astype(np.int64) + 1
    rv = a.indices.astype(np.int64) + 1
    nz = np.ascontiguousarray(a.data, dtype=np.float64)
    h = ctypes.c_void_p()
    t = time.perf_counter()
    if L.acg_approxchol(ctypes.c_int64(n), ptr(cp), ptr(rv), ptr(nz), ptr(state), ctypes.byref(h)) != 0:
        raise RuntimeError(L.acg_last_error().decode())
    factor_s = time.perf_counter() - t
    nn, F = ctypes.c_int64(), ctypes.c_int64()
    L.acg_factor_dims(h, ctypes.byref(nn), ctypes.byref(F))
    f = types.SimpleNamespace(col=np.empty(n - 1, np.int64), colptr=np.empty(n, np.int64),
                              rowval=np.empty(F.value, np.int64), fval=np.empty(F.value), d=np.empty(n))
    L.acg_factor_export(h, ptr(f.col), ptr(f.colptr), ptr(f.rowval), ptr(f.fval), ptr(f.d))
    L.acg_factor_free(h)
    f.n, f.nnz = n, F.value
    return a, f, factor_s


def rhs(n, seed):
    b = np.random.default_rng(seed).standard_normal(n)
    return b - b.mean()


def config(n, extra=None, precision="fp32 PCG in fp64 refinement"):
    c = {"workload": f"grid3({GRID_SIDE}) log-uniform weights [1e-3,1], 1 zero-mean Gaussian RHS per solve, tol 1e-8",
         "n": n, "precision": precision,
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

def cpu_solve_time(orc, b, its_hint, budget_s=25.0):
    """One-thread time of one solve of the workload with the CPU restatement.
    Runs the full solve when it fits the budget (then also returns its x and
    iteration count); otherwise times a bounded number of PCG iterations and
    scales to its_hint iterations."""
    t = time.perf_counter()
    orc(b, tol=TOL, maxits=2)
    t2 = time.perf_counter() - t
    per_it = t2 / 3.0  # the initial preconditioner application + 2 iterations
    full = per_it * (its_hint + 1)
    if full <= budget_s:
        t = time.perf_counter()
        x, its, _, _ = orc(b, tol=TOL, maxits=MAXITS)
        return time.perf_counter() - t, f"one full solve at tol 1e-8 ({its} PCG iterations, FP64)", x, its
    m = max(2, int(budget_s / per_it) - 1)
    t = time.perf_counter()
    orc(b, tol=0.0, maxits=m)
    el = time.perf_counter() - t
    return el / (m + 1) * (its_hint + 1), f"{m} FP64 PCG iterations timed, scaled to {its_hint} iterations", None, None


def _rel_centered(x, y):
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    x = x - x.mean()
    y = y - y.mean()
    return float(np.linalg.norm(x - y) / np.linalg.norm(y))


def oracle_leg(a, ldli, dev, b_cols, x_mixed, its_hint):
    """The CPU baseline leg: the oracle (the C restatement of the reference's
    pcg + LDLsolver) times one full solve of the workload on one thread, and
    checks the GPU on the same factor (outside every timed region):
      * the FP64 GPU PCG on that right-hand side against the oracle's solve at
        tol 1e-8: iteration counts and x (mean removed);
      * the mixed-precision solutions of the timed run (two of its columns)
        against the oracle's FP64 PCG to tol 1e-12."""
    import oracle as O
    orc = O.OracleSolver(a, ldli)
    t_cpu, sample, xo, ito = cpu_solve_time(orc, b_cols[0], its_hint)
    cpu = {"value": 1.0 / t_cpu, "unit": "solves/s", "cores": 1, "kind": "port", "sample": sample}
    check = {"oracle": "oracle/acg_oracle.c (FP64 pcg + LDLsolver restatement) on the same LDLinv"}
    if xo is not None:
        x64 = dev(b_cols[0], tol=TOL, maxits=MAXITS, precision="fp64")
        check["fp64_gpu_vs_oracle_tol_1e-8"] = {"gpu_its": int(dev.last_info[0].iterations), "oracle_its": int(ito),
                                               "x_rel_diff": _rel_centered(x64, xo)}
    errs = []
    for c in range(len(b_cols)):
        xe, ite, rce, _ = orc(b_cols[c], tol=1e-12, maxits=4 * MAXITS)
        errs.append({"column": c, "mixed_x_rel_error": _rel_centered(x_mixed[c], xe), "oracle_its": int(ite),
                     "oracle_true_relres": O.relres(a, xe, b_cols[c])})
    check["mixed_vs_oracle_tol_1e-12"] = errs
    return cpu, check


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
    """Max of a host float over the ranks (timings are reported as the slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_rhs_seed(rank, step, column):
    """Seed of one right-hand side: distinct for every rank, step and column
    (replicas solve disjoint work, so whole-job throughput adds up)."""
    return 1_000_000 * rank + 1000 * step + column


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
    dev = acgpu.DeviceLapSolver(a, ldli, options=json.loads(args.options) if args.options else None)
    upload_s = time.perf_counter() - t
    L = lib()
    prec = 1 if args.precision == "mixed" else 0
    k = args.rhs

    # device-resident right-hand sides: k independent columns per step, distinct per rank
    nsteps = args.warmup + args.steps
    B = torch.empty((nsteps, k, n), dtype=torch.float64, device="cuda")
    for i in range(nsteps):
        for c in range(k):
            B[i, c] = torch.from_numpy(rhs(n, rank_rhs_seed(rank, i, c)))
    X = torch.empty((k, n), dtype=torch.float64, device="cuda")
    infos = (AcgSolveInfo * k)()

    def solve_step(i, prec_override=None):
        pr = prec if prec_override is None else prec_override
        if k == 1:
            rc = L.acg_solve_device(dev._h, ctypes.c_void_p(B[i].data_ptr()), ctypes.c_void_p(X.data_ptr()), TOL,
                                    MAXITS, float("inf"), 5, pr, infos)
        else:
            rc = L.acg_solve_batch_device(dev._h, ctypes.c_void_p(B[i].data_ptr()), ctypes.c_void_p(X.data_ptr()),
                                          k, n, TOL, MAXITS, float("inf"), 5, pr, infos)
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

    # the mixed solutions of the last timed step, checked against the oracle below
    X_last = X.clone()
    last = nsteps - 1

    # the plain FP64 GPU path on the same batched workload (device-resident
    # right-hand sides, the same steps): the metric's "mixed vs FP64" arm
    fp64 = None
    if not args.no_extras:
        fsteps = min(args.steps, 3)
        solve_step(0, prec_override=0)  # captures the FP64 graphs
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record()
        fres = []
        for i in range(args.warmup, args.warmup + fsteps):
            fres += solve_step(i, prec_override=0)
        f1.record()
        torch.cuda.synchronize()
        fms = max_over_ranks(f0.elapsed_time(f1), world)
        fbad = [r for r in fres if r[3] != 0 or r[2] > TOL]
        fp64 = {"solves_per_s": world * fsteps * k / (fms * 1e-3), "steps": fsteps, "ms_per_step": fms / fsteps,
                "pcg_iterations_mean": float(np.mean([r[0] for r in fres])),
                "true_relres_max": float(max(r[2] for r in fres)), "all_converged": not fbad}

    # end to end: pinned host blocks through the asynchronous C entry
    # (acg_solve_async / acg_wait), every step's H2D and D2H inside the timed
    # region; two requests in flight, so one step's copies overlap the
    # previous step's solve
    hb = torch.empty((args.steps, k, n), dtype=torch.float64, pin_memory=True)
    hx = torch.empty((2, k, n), dtype=torch.float64, pin_memory=True)
    hb_np = hb.numpy()
    for i in range(args.steps):
        for c in range(k):
            hb_np[i, c] = rhs(n, 5_000_000 + 1_000_000 * rank + 1000 * i + c)
    e2e_bad = []

    def submit(i):
        req = ctypes.c_void_p()
        check(L.acg_solve_async(dev._h, hb[i].data_ptr(), hx[i % 2].data_ptr(), k, n, TOL, MAXITS, float("inf"), 5,
                                prec, ctypes.byref(req)))
        return req

    def finish(req):
        check(L.acg_wait(req, infos))
        e2e_bad.extend(c for c in range(k) if infos[c].status != 0 or infos[c].true_relres > TOL)

    for req in [submit(0), submit(min(1, args.steps - 1))]:  # builds both slots' graphs
        finish(req)
    e2e_bad.clear()
    barrier(world)
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record()
    inflight = []
    for i in range(args.steps):
        inflight.append(submit(i))
        if len(inflight) == 2:
            finish(inflight.pop(0))
    while inflight:
        finish(inflight.pop(0))
    e3.record()
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(e2.elapsed_time(e3), world)
    if e2e_bad:
        raise RuntimeError(f"{len(e2e_bad)} end-to-end solves missed the tolerance")

    # one right-hand side alone: latency of a single solve
    single = []
    for i in range(3):
        t0 = time.perf_counter()
        check(L.acg_solve_device(dev._h, ctypes.c_void_p(B[i, 0].data_ptr()), ctypes.c_void_p(X.data_ptr()), TOL,
                                 MAXITS, float("inf"), 5, prec, infos))
        single.append(infos[0].solve_ms)

    # roofline of the dominant kernel (the longer LDLinv sweep), timed live
    kt = dev.time_kernels_batch(k, args.precision, reps=5) if k > 1 else dev.time_kernels(args.precision, reps=5)
    stats = dev.stats()
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    # the dominant kernel: the longer of the two sweep kernels (the dense tail
    # products are timed apart and reported beside it)
    direction = "forward" if kt["forward_sweep_ms"] >= kt["backward_sweep_ms"] else "backward"
    sweep_ms = kt[direction + "_sweep_ms"]
    sweep_bytes = kt[direction + "_sweep_bytes"]
    achieved = sweep_bytes / (sweep_ms * 1e-3) / 1e9
    swept_levels = int(stats["levels"] - stats["dense_levels"])
    traffic = None
    prof = ROOT / "profiles" / (f"kb_sweep_{direction}_grid3_100_k64.md" if k > 1
                                else f"k_sweep_{direction}_grid3_100.md")
    if prof.exists() and GRID_SIDE == 100:
        import re
        m = re.search(r"dram_bytes_per_launch:\s*(\d+)", prof.read_text())
        traffic = int(m.group(1)) if m else None

    # our kernel launches per step: set-up/wrap-up 3; per refinement the
    # outer kernels (6) and one preconditioner application (forward and
    # backward launches); per inner iteration the library's count
    per_it = kt["launches_per_iteration"]
    per_ref = 6 + 2 * kt["forward_launches"]
    launches = args.steps * (3 + refs.max() * per_ref + its.max() * per_it)

    extras = {}
    if not args.no_extras:
        extras = run_extras(args, rank, world)

    if rank == 0:
        cpu = None
        oracle_check = None
        if world == 1 and not args.no_cpu:
            ncheck = min(2, k)
            b_cols = [B[last, c].cpu().numpy() for c in range(ncheck)]
            x_mixed = [X_last[c].cpu().numpy() for c in range(ncheck)]
            cpu, oracle_check = oracle_leg(a, ldli, dev, b_cols, x_mixed, int(round(its.mean())))
        value = world * args.steps * k / (ms * 1e-3)
        kern = (f"kb_sweep<float,{k // 8 if k >= 8 else 1},{direction}> (batched LDLinv {direction} sweep, {k} columns)"
                if k > 1 else f"k_sweep<float,{direction}> (LDLinv {direction} sweep)")
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (SpMV, sweeps) / f64 (residual, dots, correction)"
            if prec == 1 else "f64", "data": "synthetic (seeded grid weights and Gaussian RHS)",
            "config": config(n, {"parallelism": f"replicas x{world}", "rhs_per_step": k,
                                 "solver_options": json.loads(args.options) if args.options else {},
                                 "batching": f"{k} independent single-RHS solves per step in one batched launch",
                                 "pcg_iterations_mean": float(its.mean()), "refinements_mean": float(refs.mean()),
                                 "true_relres_max": float(res.max()), "factor_s": factor_s, "upload_s": upload_s,
                                 "levels": stats["levels"], "factor_nnz": stats["nnz_factor"]}),
            "fp64_batched": fp64,
            "mixed_over_fp64": (value / fp64["solves_per_s"]) if fp64 else None,
            "oracle_check": oracle_check,
            **extras,
            "single_rhs": {"latency_ms": float(np.median(single)), "solves_per_s": 1e3 / float(np.median(single))},
            "e2e": {"value": world * args.steps * k / (e2e_ms * 1e-3), "unit": "solves/s",
                    "h2d_bytes_per_step": 8 * n * k, "d2h_bytes_per_step": 8 * n * k},
            "roofline": {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                         "algorithmic_bytes_per_launch": sweep_bytes, "launch_ms": sweep_ms,
                         "forward_sweep_ms": kt["forward_sweep_ms"], "backward_sweep_ms": kt["backward_sweep_ms"],
                         "dense_tail_ms": kt["dense_ms"], "dense_tail_vertices": stats["dense_vertices"],
                         # the sweep walks the DAG's head levels one after another: time per level
                         "swept_levels": swept_levels, "us_per_level": 1e3 * sweep_ms / max(1, swept_levels),
                         "spmv_ms": kt["spmv_ms"], "spmv_gbs": kt["spmv_bytes"] / (kt["spmv_ms"] * 1e-3) / 1e9},
            # every kernel of a batched solve, each timed alone (CUDA events, ms per launch)
            "kernel_ms": ({key: round(kt[key + "_ms"], 4) for key in
                           ("spmv", "forward_sweep", "backward_sweep", "dense", "pq", "update", "yzr", "pupdate",
                            "gather", "scatter", "true_residual")} if k > 1 else None),
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": int(round(launches)),
        }
        print(json.dumps(line), flush=True)
    dev.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---- the other workloads of the solve phase (reported, not the headline) -------

def _device_solve(dev, b, prec, tol, maxits=MAXITS):
    x = dev(b, tol=tol, maxits=maxits, precision=prec)
    return x, dev.last_info[0]


def run_grid2_200(args):
    """grid2(200), unit weights, one zero-mean Gaussian RHS, tol 1e-6: FP64 on the
    GPU against the CPU restatement on the same LDLinv."""
    import acgpu
    import oracle as O
    from acgpu import generators as G
    a = G.grid2(200)
    acgpu.seed(FACTOR_SEED)
    ldli = acgpu.approx_chol(a)
    dev = acgpu.DeviceLapSolver(a, ldli)
    b = rhs(a.shape[0], 11)
    for _ in range(3):
        x, info = _device_solve(dev, b, "fp64", 1e-6)
    orc = O.OracleSolver(a, ldli)
    t = time.perf_counter()
    xo, ito, rco, _ = orc(b, tol=1e-6, maxits=1000)
    t_cpu = time.perf_counter() - t
    diff = float(np.linalg.norm(O.center(x) - O.center(xo)) / np.linalg.norm(O.center(xo)))
    print(json.dumps({"workload": "grid2(200) unit weights, tol 1e-6, fp64", "n": a.shape[0],
                      "gpu_ms": info.solve_ms, "gpu_its": info.iterations, "gpu_relres": O.relres(a, x, b),
                      "cpu_port_ms": t_cpu * 1e3, "cpu_its": ito, "cpu_relres": O.relres(a, xo, b),
                      "x_rel_diff_vs_cpu": diff, "levels": dev.stats()["levels"]}), flush=True)
    dev.close()


def run_matchings_2m(args):
    """Path over a random permutation + 4 random perfect matchings, n = 2M,
    lognormal(0, 2) weights; mixed precision to 1e-8; level count and LDLinv GB/s."""
    n = 2_000_000 if GRID_SIDE == 100 else GRID_SIDE ** 3
    print(json.dumps(matchings_2m_record(n)), flush=True)


def run_orderings(args):
    """The four elimination orders of approxchol_lap (:deg, :given, :wdeg,
    :random; src/approxChol.jl:1628-1789) on grid3(50) with log-uniform weights:
    factor size, DAG depth (what bounds the sweeps), factor and solve time."""
    import acgpu
    from acgpu import generators as G
    side = 50
    a = G.grid3(side, weights="loguniform", seed=7)
    n = a.shape[0]
    b = rhs(n, 13)
    out = {"workload": f"elimination orders on grid3({side}) log-uniform weights, tol 1e-8", "n": n}
    for order in ("deg", "lap2", "wdeg", "random", "given"):
        # lap2: the split/merge elimination of approxchol_lap2 (:deg, split = merge = 2)
        params = acgpu.ApproxCholParams("deg", 5, 2, 2) if order == "lap2" else acgpu.ApproxCholParams(order=order)
        acgpu.seed(FACTOR_SEED)
        t = time.perf_counter()
        ldli = acgpu.approx_chol(a, params)
        factor_s = time.perf_counter() - t
        dev = acgpu.DeviceLapSolver(a, ldli, params=params)
        st = dev.stats()
        row = {"factor_s": factor_s, "factor_nnz": ldli.nnz, "levels": st["levels"],
               "dense_tail_levels": st["dense_levels"]}
        # the given order's DAG is far deeper (the slowest solve, as the
        # reference documents): one mixed solve of it is enough
        for prec in (("mixed",) if order == "given" else ("mixed", "fp64")):
            for _ in range(1 if order == "given" else 2):
                x, info = _device_solve(dev, b, prec, TOL)
            row[prec] = {"solve_ms": info.solve_ms, "its": info.iterations, "refinements": info.refinements,
                         "true_relres": info.true_relres, "status": info.status}
        out[order] = row
        dev.close()
    print(json.dumps(out), flush=True)


def run_grid3_64rhs(args):
    """64 right-hand sides on the 1M weighted 3D grid: FP64 batched vs mixed batched."""
    import torch
    import acgpu
    from acgpu._lib import AcgSolveInfo, check, lib
    a, ldli, factor_s = build_workload()
    n = a.shape[0]
    dev = acgpu.DeviceLapSolver(a, ldli)
    k = 64
    B = torch.empty((k, n), dtype=torch.float64, device="cuda")
    for c in range(k):
        B[c] = torch.from_numpy(rhs(n, 77 + c))
    X = torch.empty_like(B)
    infos = (AcgSolveInfo * k)()
    out = {"workload": "64 RHS on grid3(100) log-uniform weights, tol 1e-8", "n": n}
    for prec, name in ((0, "fp64"), (1, "mixed")):
        times = []
        for rep in range(3):
            torch.cuda.synchronize()
            t = time.perf_counter()
            check(lib().acg_solve_batch_device(dev._h, ctypes.c_void_p(B.data_ptr()), ctypes.c_void_p(X.data_ptr()),
                                               k, n, TOL, MAXITS, float("inf"), 5, prec, infos))
            times.append(time.perf_counter() - t)
        its = [infos[c].iterations for c in range(k)]
        out[name] = {"solves_per_s": k / min(times), "batch_ms": 1e3 * min(times), "its_mean": float(np.mean(its)),
                     "true_relres_max": max(infos[c].true_relres for c in range(k))}
        kt = dev.time_kernels_batch(k, name, reps=3)
        out[name]["forward_ms"] = kt["forward_ms"]
        out[name]["ldlinv_forward_gbs"] = kt["forward_bytes"] / (kt["forward_ms"] * 1e-3) / 1e9
    out["mixed_over_fp64"] = out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"]
    print(json.dumps(out), flush=True)
    dev.close()


def run_sweep_levels(args):
    """The 64-column FP32 sweeps of the headline workload cut after a range of
    levels (acg_time_sweep_levels): how the sweep time splits over the
    dependency DAG's levels.  Not a bench line: one JSON object with the points
    and the per-level cost between them."""
    import acgpu
    a, ldli, _ = build_workload()
    dev = acgpu.DeviceLapSolver(a, ldli)
    st = dev.stats()
    swept = int(st["levels"] - st["dense_levels"])
    pts = sorted({0, 1, 2, 5, 10, 20, 50, 100, 150, 200, 250, 300, 350, 400} | {max(swept - 1, 0)})
    pts = [p for p in pts if p < swept]
    rows = dev.time_sweep_levels(pts, nrhs=args.rhs, precision=args.precision, reps=5)
    for i, r in enumerate(rows):
        if i + 1 < len(rows):
            nxt = rows[i + 1]
            span = nxt["level"] - r["level"]
            # forward: levels (L, L'] cost f(L') - f(L); backward: levels [L, L')
            r["forward_us_per_level_next"] = 1e3 * (nxt["forward_ms"] - r["forward_ms"]) / span
            r["backward_us_per_level_next"] = 1e3 * (r["backward_ms"] - nxt["backward_ms"]) / span
    out = {"workload": f"grid3({GRID_SIDE}) log-uniform weights, {args.rhs} columns, {args.precision}",
           "levels": int(st["levels"]), "swept_levels": swept, "dense_levels": int(st["dense_levels"]),
           "points": rows}
    print(json.dumps(out), flush=True)
    dev.close()


def run_many_graphs(args):
    """256 graphs in one launch: half 2D grids with side uniform in [32, 256],
    half random geometric graphs (n uniform in [1e3, 1e5], mean degree 8,
    weights 1/distance), one right-hand side each, tol 1e-8.  A random
    geometric graph may be disconnected: as approxchol_lap does
    (lapWrapComponents, src/solverInterface.jl:212-275), each component of at
    least 50 vertices is its own PCG system in the one group launch, smaller
    ones are solved on the host and singletons get zero.  FP64 and mixed
    precision, against the same graphs solved one after another."""
    import acgpu
    from acgpu import generators as G
    from acgpu.solvers import _DenseGroundedSolver
    rng = np.random.default_rng(44)
    graphs = []
    for i in range(args.group_graphs):
        s_ = int(rng.integers(1 << 30))
        if i % 2 == 0:
            graphs.append(G.grid2(int(rng.integers(32, 257)), weights="loguniform", seed=s_))
        else:
            graphs.append(G.random_geometric(int(rng.integers(1000, 100001)), seed=s_))
    # split every graph into components: members of the group, host solves, singletons
    members, small, nsingle = [], [], 0
    for gi, a in enumerate(graphs):
        co = acgpu.components(a)
        for ind in acgpu.vec_to_comps(co):
            if len(ind) == 1:
                nsingle += 1
            elif len(ind) < 50:
                small.append((gi, ind))
            else:
                members.append((gi, ind))
    comp_graphs = [acgpu.solvers._csc(graphs[gi][ind][:, ind]) for gi, ind in members]
    t = time.perf_counter()
    factors = []
    for i, a in enumerate(comp_graphs):
        acgpu.seed(500 + i)
        factors.append(acgpu.approx_chol(a))
    factor_s = time.perf_counter() - t
    t = time.perf_counter()
    gs = acgpu.GroupSolver(comp_graphs, factors)
    upload_s = time.perf_counter() - t
    small_solvers = [_DenseGroundedSolver(graphs[gi][ind][:, ind]) for gi, ind in small]
    bs = [rhs(a.shape[0], 900 + i) for i, a in enumerate(graphs)]
    # per component: b restricted and centred (the solvable part, as blockSolver solves it)
    comp_b = [bs[gi][ind] - bs[gi][ind].mean() for gi, ind in members]
    small_b = [bs[gi][ind] - bs[gi][ind].mean() for gi, ind in small]
    out = {"workload": f"{len(graphs)} graphs in one launch (2D grids side U[32,256], RGG n U[1e3,1e5] with all "
                       "their components), 1 RHS each, tol 1e-8",
           "n_total": int(sum(a.shape[0] for a in graphs)), "group_members": len(members),
           "host_small_components": len(small), "singletons": nsingle, "factor_s": factor_s, "upload_s": upload_s}
    for prec in ("fp64", "mixed"):
        times = []
        for rep in range(3):
            t = time.perf_counter()
            xs = gs(comp_b, tol=TOL, maxits=MAXITS, precision=prec)
            for sv, b in zip(small_solvers, small_b):
                sv(b)
            times.append(time.perf_counter() - t)
        infos = gs.last_info
        out[prec] = {"group_ms": 1e3 * min(times), "graphs_per_s": len(graphs) / min(times),
                     "its_max": max(i.iterations for i in infos),
                     "its_mean": float(np.mean([i.iterations for i in infos])),
                     "true_relres_max": max(i.true_relres for i in infos),
                     "all_converged": all(i.status == 0 for i in infos)}
        its_by_prec = out.setdefault("_its", {})
        its_by_prec[prec] = [(int(i.iterations), int(i.refinements), int(i.status)) for i in infos]
    # the group waits for its slowest member: the five with the most iterations
    # in each precision, with the member's size and weight spread
    slow = {}
    for prec in ("fp64", "mixed"):
        order = sorted(range(len(members)), key=lambda m: -out["_its"][prec][m][0])[:5]
        slow[prec] = [{"member": m, "n": int(comp_graphs[m].shape[0]),
                       "weight_max_over_min": float(comp_graphs[m].data.max() / comp_graphs[m].data.min()),
                       "fp64_its": out["_its"]["fp64"][m][0],
                       "mixed_its": out["_its"]["mixed"][m][0], "mixed_refinements": out["_its"]["mixed"][m][1]}
                      for m in order]
    out["slowest_members"] = slow
    del out["_its"]
    out["levels_max"] = gs.stats()["levels"]
    if args.tune:
        # config 4b's tuned tiles: one round of coordinate descent over the
        # union sweeps' knobs, measured by the FP64 group solve itself
        from acgpu.tuning import coordinate_descent

        def group_ms(opts):
            g = acgpu.GroupSolver(comp_graphs, factors, options={k: v for k, v in opts.items() if v != 0})
            try:
                ts = []
                for _ in range(2):
                    t0 = time.perf_counter()
                    g(comp_b, tol=TOL, maxits=MAXITS, precision="fp64")
                    ts.append(time.perf_counter() - t0)
                return 1e3 * min(ts)
            finally:
                g.close()

        space = {"sweep_heavy": [0, 8, 32], "sweep_blocks_per_sm": [0, 2, 3], "poll_mode": [0, 1, 2]}
        tr = coordinate_descent(group_ms, space, rounds=1, min_gain=0.02)
        out["tuned_fp64"] = {"options": tr.options, "group_ms": tr.ms, "default_ms": tr.baseline_ms,
                             "trials": [(o, round(ms, 2)) for o, ms in tr.trials]}
    seq = []
    for a, f, b in zip(comp_graphs, factors, comp_b):
        dev = acgpu.DeviceLapSolver(a, f)
        dev(b, tol=TOL, maxits=MAXITS)
        dev(b, tol=TOL, maxits=MAXITS)
        seq.append(dev.last_info[0].solve_ms)
        dev.close()
    out["sequential_fp64_ms"] = float(sum(seq))
    out["speedup_fp64"] = float(sum(seq)) / out["fp64"]["group_ms"]
    print(json.dumps(out), flush=True)
    gs.close()


def serving_graph_pool(count, seed):
    """Graphs for the serving stream: 2D/3D grids, path + random matchings and
    random geometric graphs (whole, components and all), n log-uniform in
    [1e3, 1e6], lognormal(0, 1) weights."""
    from acgpu import generators as G
    rng = np.random.default_rng(seed)
    fams = ["grid2", "grid3", "matchings", "rgg"]
    pool = []
    for i in range(count):
        fam = fams[i % 4]
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
        s = int(rng.integers(1 << 30))
        if fam == "grid2":
            side = max(2, int(round(np.sqrt(n))))
            a = G.grid2(side, weights="lognormal:1", seed=s)
        elif fam == "grid3":
            side = max(2, int(round(n ** (1 / 3))))
            a = G.grid3(side, weights="lognormal:1", seed=s)
        elif fam == "matchings":
            a = G.path_plus_matchings(max(4, n - n % 2), k=4, sigma=1.0, seed=s)
        else:
            # the whole graph: a disconnected one is served per component
            a = G.random_geometric(n, seed=s, weights="lognormal:1")
        pool.append((f"{fam}-{a.shape[0]}", a))
    return pool


def serve_stream(pool, factors, nreq, rate, hbm_gb, seed=7):
    """One Poisson stream of nreq requests (1-16 right-hand sides each, tol
    1e-8) over the cached graphs of pool, served twice: continuous batching in
    mixed precision, and the unbatched FP64 GPU path (one request at a time,
    one right-hand side per solve).  Returns the latency/throughput record of
    each."""
    from acgpu.serving import SolveServer
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
    picks = rng.integers(len(pool), size=nreq)
    ks = rng.integers(1, 17, size=nreq)
    rhs_blocks = [np.random.default_rng(10_000 + r).standard_normal((pool[picks[r]][1].shape[0], int(ks[r])))
                  for r in range(nreq)]
    results = {}
    for label, kw in (("batched_mixed", dict(precision="mixed", slots=64)),
                      ("unbatched_fp64", dict(precision="fp64", unbatched=True))):
        server = SolveServer(hbm_budget=int(hbm_gb * (1 << 30)), **kw)
        for i, (gid, a) in enumerate(pool):
            server.register(gid, a, ldli=factors[gid], seed=None if factors[gid] is not None else 3000 + i)
        with server:
            for gid, a in pool:  # warm: upload and capture every graph once
                server.submit(gid, np.random.default_rng(1).standard_normal(a.shape[0]), tol=TOL).result()
            server.completed.clear()
            futs = []
            t0 = time.perf_counter()
            for r in range(nreq):
                delay = t0 + arrivals[r] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                futs.append(server.submit(pool[picks[r]][0], rhs_blocks[r], tol=TOL))
            worst = 0.0
            for f in futs:
                X, infos = f.result()
                worst = max(worst, max(i.true_relres for i in infos))
            st = server.latency_stats()
            st["true_relres_max"] = worst
            results[label] = st
    results["speedup_solves_per_s"] = (results["batched_mixed"]["solves_per_s"] /
                                       results["unbatched_fp64"]["solves_per_s"])
    return results


def factor_pool(pool, seed0):
    """Host factors of the pool's connected graphs (a disconnected graph is
    factored per component when the server registers it: None here)."""
    import acgpu
    factors = {}
    t = time.perf_counter()
    for i, (gid, a) in enumerate(pool):
        acgpu.seed(seed0 + i)
        factors[gid] = acgpu.approx_chol(a) if acgpu.components(a).max() == 1 else None
    return factors, time.perf_counter() - t


def run_serving(args):
    """Poisson stream of solve requests over a pool of cached graphs, 1-16
    right-hand sides each, tol 1e-8: continuous batching (mixed precision)
    against the unbatched FP64 GPU path (one request at a time, one RHS per solve)."""
    pool = serving_graph_pool(args.serving_graphs, seed=2024)
    factors, factor_s = factor_pool(pool, 1000)
    results = serve_stream(pool, factors, args.serving_requests, args.serving_rate, args.serving_hbm_gb)
    out = {"workload": "serving: Poisson arrivals, graphs from 2D/3D grids, matchings, RGG, "
                       "n log-uniform [1e3,1e6], lognormal(0,1) weights, 1-16 RHS, tol 1e-8",
           "graphs": [(gid, int(a.shape[0])) for gid, a in pool], "requests": args.serving_requests,
           "arrival_rate_per_s": args.serving_rate, "factor_s_total": factor_s, **results}
    print(json.dumps(out), flush=True)


def matchings_2m_record(n=2_000_000):
    """The 2,000,000-vertex path + 4 random perfect matchings graph
    (lognormal(0, 2) weights): DAG level count, LDLinv sweep bandwidth and one
    mixed and one FP64 solve to tol 1e-8 (one right-hand side)."""
    import acgpu
    from acgpu import generators as G
    a = G.path_plus_matchings(n, k=4, sigma=2.0, seed=3)
    acgpu.seed(FACTOR_SEED)
    t = time.perf_counter()
    ldli = acgpu.approx_chol(a)
    factor_s = time.perf_counter() - t
    dev = acgpu.DeviceLapSolver(a, ldli)
    b = rhs(n, 12)
    out = {"workload": f"path + 4 random matchings, n={n}, lognormal(0,2) weights, 1 RHS, tol 1e-8", "n": n,
           "avg_degree": a.nnz / n, "factor_nnz": ldli.nnz, "factor_s": factor_s, "levels": dev.stats()["levels"]}
    for prec in ("mixed", "fp64"):
        for _ in range(2):
            x, info = _device_solve(dev, b, prec, TOL)
        kt = dev.time_kernels(prec, reps=3)
        out[prec] = {"solve_ms": info.solve_ms, "its": info.iterations, "refinements": info.refinements,
                     "true_relres": info.true_relres, "status": info.status,
                     "forward_ms": kt["forward_ms"], "backward_ms": kt["backward_ms"],
                     "ldlinv_forward_gbs": kt["forward_bytes"] / (kt["forward_ms"] * 1e-3) / 1e9,
                     "ldlinv_backward_gbs": kt["backward_bytes"] / (kt["backward_ms"] * 1e-3) / 1e9}
    dev.close()
    return out


def run_extras(args, rank, world):
    """The rest of the metric, beside the headline (N = 1 only; each takes
    seconds): serving p50/p99 on a short Poisson stream, the 2M
    path+matchings graph's level count and LDLinv GB/s, and the solve with the
    opt-in parallel elimination's factor."""
    if world > 1 or rank != 0:
        return {}
    out = {}
    pool = serving_graph_pool(8, seed=2024)
    factors, factor_s = factor_pool(pool, 1000)
    t = time.perf_counter()
    res = serve_stream(pool, factors, 100, 40.0, args.serving_hbm_gb)
    out["serving"] = {"workload": "100 requests, Poisson 40/s, 8 cached graphs (2D/3D grids, matchings, RGG, "
                                  "n log-uniform [1e3,1e6], lognormal(0,1) weights), 1-16 RHS each, tol 1e-8",
                      "graphs": [(gid, int(a.shape[0])) for gid, a in pool], "factor_s_total": factor_s,
                      "wall_s": time.perf_counter() - t, **res}
    out["path_matchings_2m"] = matchings_2m_record()
    out["parallel_factor"] = parallel_factor_record()
    return out


def parallel_factor_record(k=64, steps=3):
    """The opt-in parallel elimination (acgpu.approx_chol_parallel; not the
    reference's, a different random sample) on the same 1M grid: host time on
    all cores, rounds, the DAG depth the GPU sweeps walk, and the 64-column
    mixed solve rate with that factor (device-resident right-hand sides)."""
    import torch
    import acgpu
    from acgpu import generators as G
    from acgpu._lib import AcgSolveInfo, check, lib
    a = G.grid3(GRID_SIDE, weights="loguniform", seed=WEIGHT_SEED)
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    t = time.perf_counter()
    ldli, rounds = acgpu.approx_chol_parallel(a, seed=FACTOR_SEED, threads=threads)
    factor_s = time.perf_counter() - t
    n = a.shape[0]
    dev = acgpu.DeviceLapSolver(a, ldli)
    st = dev.stats()
    B = torch.empty((steps + 1, k, n), dtype=torch.float64, device="cuda")
    for i in range(steps + 1):
        for c in range(k):
            B[i, c] = torch.from_numpy(rhs(n, 7_000_000 + 1000 * i + c))
    X = torch.empty((k, n), dtype=torch.float64, device="cuda")
    infos = (AcgSolveInfo * k)()
    res = []
    for i in range(steps + 1):
        if i == 1:
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
        check(lib().acg_solve_batch_device(dev._h, ctypes.c_void_p(B[i].data_ptr()), ctypes.c_void_p(X.data_ptr()),
                                           k, n, TOL, MAXITS, float("inf"), 5, 1, infos))
        if i >= 1:
            res += [(infos[c].iterations, infos[c].true_relres, infos[c].status) for c in range(k)]
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    kt = dev.time_kernels_batch(k, "mixed", reps=3)
    # one right-hand side alone: the shallower DAG shortens every sweep
    single = []
    for i in range(3):
        check(lib().acg_solve_device(dev._h, ctypes.c_void_p(B[0, i].data_ptr()), ctypes.c_void_p(X.data_ptr()), TOL,
                                     MAXITS, float("inf"), 5, 1, infos))
        single.append(infos[0].solve_ms)
    dev.close()
    return {"workload": f"grid3({GRID_SIDE}) log-uniform weights, factor by the opt-in parallel elimination, "
                        f"{k} RHS per batched mixed solve, tol 1e-8",
            "factor_s": factor_s, "threads": threads, "rounds": rounds, "factor_nnz": ldli.nnz,
            "levels": st["levels"], "dense_levels": st["dense_levels"],
            "solves_per_s": steps * k / (ms * 1e-3), "pcg_iterations_mean": float(np.mean([r[0] for r in res])),
            "true_relres_max": float(max(r[1] for r in res)), "all_converged": all(r[2] == 0 for r in res),
            "forward_sweep_ms": kt["forward_sweep_ms"], "backward_sweep_ms": kt["backward_sweep_ms"],
            "single_rhs_latency_ms": float(np.median(single))}


def run_reference(args):
    """The reference's solve on the host cores: the CPU restatement of pcg +
    LDLsolver (oracle port), one independent solve per thread."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import oracle as O
    a, ldli, factor_s = build_workload_host_only()
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
            "config": config(n, {"parallelism": f"{threads} host threads", "factor_s": factor_s},
                             precision="fp64 PCG (CPU restatement of the reference's solve)"),
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
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg (and its oracle check)")
    ap.add_argument("--options", default="", help="acg_options knobs as JSON (tuning), e.g. '{\"level_order\": 1}'")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the extra keys (FP64 arm, serving latency, 2M path+matchings graph)")
    ap.add_argument("--side", type=int, default=GRID_SIDE, help="grid side (100 = the benchmark workload)")
    ap.add_argument("--rhs", type=int, default=64, help="independent right-hand sides per step (batched)")
    ap.add_argument("--workload", default="grid3",
                    choices=["grid3", "grid2_200", "matchings_2m", "grid3_64rhs", "many_graphs", "serving", "orderings",
                             "sweep_levels"],
                    help="grid3 = the headline line; the others report the remaining workloads")
    ap.add_argument("--serving-graphs", type=int, default=16)
    ap.add_argument("--group-graphs", type=int, default=256)
    ap.add_argument("--serving-requests", type=int, default=300)
    ap.add_argument("--serving-rate", type=float, default=40.0, help="requests per second")
    ap.add_argument("--serving-hbm-gb", type=float, default=120.0)
    ap.add_argument("--tune", action="store_true", help="many_graphs: tune the group's sweep knobs first")
    args = ap.parse_args()
    globals()["GRID_SIDE"] = args.side
    if args.warmup < 3 and args.impl == "acgpu":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "grid3":
        run_acgpu(args)
    else:
        import torch
        torch.cuda.init()
        {"orderings": run_orderings, "grid2_200": run_grid2_200, "matchings_2m": run_matchings_2m, "grid3_64rhs": run_grid3_64rhs, "many_graphs": run_many_graphs,
         "serving": run_serving, "sweep_levels": run_sweep_levels}[args.workload](args)


if __name__ == "__main__":
    main()
