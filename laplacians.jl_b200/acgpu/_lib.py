"""ctypes binding of libacgpu.so (declarations in include/acgpu.h).

The library is required: importing a solver entry point without it raises,
there is no CPU substitute for the device path.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(os.environ.get("ACGPU_LIB", Path(__file__).resolve().parent / "libacgpu.so"))

ACG_OK = 0
STOP_NAMES = {
    0: "converged", 1: "maxits", 2: "stagnation |p|", 3: "stagnation |q|", 4: "rho stagnation",
    5: "inf", 6: "stagnation beta|p|", 7: "maxtime",
}
ERR_NAMES = {-1: "invalid", -2: "out of memory", -3: "cuda", -4: "device wait timeout", -5: "no device",
             -6: "admission refused"}

i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


class AcgOptions(ctypes.Structure):
    _fields_ = [("sweep_lanes", ctypes.c_int), ("spmv_lanes", ctypes.c_int), ("wide_level_min", ctypes.c_int),
                ("sweep_blocks_per_sm", ctypes.c_int), ("poll_mode", ctypes.c_int), ("tail", ctypes.c_int),
                ("batch_bwd_heavy", ctypes.c_int), ("batch_fwd_heavy", ctypes.c_int),
                ("batch_blocks_per_sm", ctypes.c_int), ("sweep_heavy", ctypes.c_int),
                ("dense_tail", ctypes.c_int), ("sweep_stride", ctypes.c_int),
                ("level_order", ctypes.c_int), ("spin_limit", ctypes.c_int),
                ("test_unproduced_task", ctypes.c_int), ("min_inner_tol", ctypes.c_double)]


class AcgStats(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("nnz_lap", ctypes.c_int64), ("nnz_factor", ctypes.c_int64),
                ("levels", ctypes.c_int64), ("wide_levels", ctypes.c_int64), ("thin_runs", ctypes.c_int64),
                ("sweep_lanes", ctypes.c_int), ("spmv_lanes", ctypes.c_int), ("device_bytes", ctypes.c_int64),
                ("batch_capacity", ctypes.c_int64), ("tail_levels", ctypes.c_int64),
                ("tail_vertices", ctypes.c_int64), ("dense_levels", ctypes.c_int64),
                ("dense_vertices", ctypes.c_int64)]


class AcgSolveInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("refinements", ctypes.c_int64), ("relres", ctypes.c_double),
                ("best_relres", ctypes.c_double), ("true_relres", ctypes.c_double), ("solve_ms", ctypes.c_double),
                ("status", ctypes.c_int), ("levels", ctypes.c_int)]


class AcgKernelTimes(ctypes.Structure):
    _fields_ = [("spmv_ms", ctypes.c_double), ("forward_ms", ctypes.c_double), ("backward_ms", ctypes.c_double),
                ("iteration_ms", ctypes.c_double), ("launches_per_iteration", ctypes.c_int),
                ("forward_launches", ctypes.c_int), ("spmv_bytes", ctypes.c_double),
                ("forward_bytes", ctypes.c_double), ("backward_bytes", ctypes.c_double),
                ("forward_sweep_ms", ctypes.c_double), ("backward_sweep_ms", ctypes.c_double),
                ("dense_ms", ctypes.c_double), ("forward_sweep_bytes", ctypes.c_double),
                ("backward_sweep_bytes", ctypes.c_double), ("dense_bytes", ctypes.c_double),
                ("pq_ms", ctypes.c_double), ("update_ms", ctypes.c_double), ("yzr_ms", ctypes.c_double),
                ("pupdate_ms", ctypes.c_double), ("pq_bytes", ctypes.c_double), ("update_bytes", ctypes.c_double),
                ("yzr_bytes", ctypes.c_double), ("pupdate_bytes", ctypes.c_double),
                ("gather_ms", ctypes.c_double), ("scatter_ms", ctypes.c_double), ("true_residual_ms", ctypes.c_double)]


# (name, restype, argtypes) for every entry point of include/acgpu.h
SIGNATURES = [
    ("acg_last_error", ctypes.c_char_p, []),
    ("acg_rng_seed", ctypes.c_int, [ctypes.c_uint64, u64p]),
    ("acg_rng_rand", ctypes.c_int, [u64p, f64p, ctypes.c_int64]),
    ("acg_sha256", ctypes.c_int, [u8p, ctypes.c_int64, u8p]),
    ("acg_approxchol", ctypes.c_int, [ctypes.c_int64, i64p, i64p, f64p, u64p, ctypes.POINTER(ctypes.c_void_p)]),
    ("acg_approxchol_ordered", ctypes.c_int, [ctypes.c_int64, i64p, i64p, f64p, ctypes.c_void_p, u64p,
                                               ctypes.POINTER(ctypes.c_void_p)]),
    ("acg_approxchol_split", ctypes.c_int, [ctypes.c_int64, i64p, i64p, f64p, ctypes.c_int64, ctypes.c_int64, u64p,
                                             ctypes.POINTER(ctypes.c_void_p)]),
    ("acg_approxchol_parallel", ctypes.c_int, [ctypes.c_int64, i64p, i64p, f64p, ctypes.c_uint64, ctypes.c_int,
                                                ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_void_p)]),
    ("acg_factor_dims", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    ("acg_factor_export", ctypes.c_int, [ctypes.c_void_p, i64p, i64p, i64p, f64p, f64p]),
    ("acg_factor_free", None, [ctypes.c_void_p]),
    ("acg_ldlinv_save", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int64, i64p, i64p, i64p, f64p, f64p,
                                       ctypes.c_int64]),
    ("acg_ldlinv_load", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("acg_device_check", ctypes.c_int, []),
    ("acg_create", ctypes.c_int, [ctypes.c_int64, i64p, i64p, f64p, i64p, i64p, i64p, f64p, f64p, ctypes.c_int64,
                                  ctypes.c_int, ctypes.POINTER(AcgOptions), ctypes.POINTER(ctypes.c_void_p)]),
    ("acg_create_group", ctypes.c_int, [ctypes.c_int64, i64p, ctypes.c_int64, i64p, i64p, f64p, i64p, ctypes.c_int64,
                                        i64p, i64p, f64p, f64p, ctypes.c_int64, ctypes.c_int,
                                        ctypes.POINTER(AcgOptions), ctypes.POINTER(ctypes.c_void_p)]),
    ("acg_solve_group", ctypes.c_int, [ctypes.c_void_p, f64p, f64p, ctypes.c_double, ctypes.c_int64, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_int, ctypes.POINTER(AcgSolveInfo)]),
    ("acg_destroy", None, [ctypes.c_void_p]),
    ("acg_solver_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AcgStats)]),
    ("acg_solve", ctypes.c_int, [ctypes.c_void_p, f64p, f64p, ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                 ctypes.c_int64, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(AcgSolveInfo)]),
    ("acg_solve_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                        ctypes.c_int64, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(AcgSolveInfo)]),
    ("acg_solve_batch_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                              ctypes.c_int64, ctypes.c_double, ctypes.c_int64, ctypes.c_double,
                                              ctypes.c_int, ctypes.c_int, ctypes.POINTER(AcgSolveInfo)]),
    ("acg_solve_async", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                       ctypes.c_int64, ctypes.c_double, ctypes.c_int64, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("acg_poll", ctypes.c_int, [ctypes.c_void_p]),
    ("acg_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AcgSolveInfo)]),
    ("acg_ldlsolve", ctypes.c_int, [ctypes.c_void_p, f64p, f64p, ctypes.c_int]),
    ("acg_lap_mul", ctypes.c_int, [ctypes.c_void_p, f64p, f64p, ctypes.c_int]),
    ("acg_time_kernels", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(AcgKernelTimes)]),
    ("acg_time_kernels_batch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.POINTER(AcgKernelTimes)]),
    ("acg_time_sweep_levels", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p]),
    ("acg_ldlsolve_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.c_void_p]),
    ("acg_serve_open", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_void_p)]),
    ("acg_serve_submit", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                        ctypes.c_int64, ctypes.c_double, ctypes.c_int64, ctypes.c_double, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_void_p)]),
    ("acg_serve_poll", ctypes.c_int, [ctypes.c_void_p]),
    ("acg_serve_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AcgSolveInfo)]),
    ("acg_serve_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(ctypes.c_int64)]),
    ("acg_serve_close", ctypes.c_int, [ctypes.c_void_p]),
]

_lib = None


class AcgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{ERR_NAMES.get(code, code)}] {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """Load libacgpu.so once; raise if it is absent (no fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"libacgpu.so not found at {LIB_PATH}; build it with laplacians.jl_b200/build.py")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> int:
    """Raise AcgError for negative status codes, pass others through."""
    if rc < 0:
        raise AcgError(rc, lib().acg_last_error().decode(errors="replace"))
    return rc
