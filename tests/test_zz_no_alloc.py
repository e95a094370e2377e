"""GPU test of the allocation-free preconditioner entry point.

acg_ldlsolve_noalloc serves callers that may not allocate device memory when
they apply the preconditioner (a serving loop running from a fixed memory
pool, a host runtime whose own allocator owns the GPU's memory, or a caller
that cannot let cudaMalloc/cudaFree synchronize the device).  It must give the same y as the
ordinary entry point acg_ldlsolve, call after call, while taking all of its
scratch from the library's fixed array.  This file is collected last so that a
run stopping at the first failure has already run every other test; it also
passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import acgpu
from acgpu import generators as G
from acgpu._lib import lib

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12  # the bar the LDLsolver parity tests use
TOL_FP32 = 1e-4


def _rel(x, y):
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


@pytest.fixture(scope="module")
def solver(gpu_ok):
    a = G.grid3(18, weights="loguniform", seed=11)
    acgpu.seed(5)
    dev = acgpu.DeviceLapSolver(a, acgpu.approx_chol(a))
    yield dev
    dev.close()


def _noalloc(dev, r, precision):
    import torch
    r_dev = torch.from_numpy(r).to("cuda")
    y_dev = torch.full_like(r_dev, float("nan"))
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib().acg_ldlsolve_noalloc(dev._h, ctypes.c_void_p(r_dev.data_ptr()), ctypes.c_void_p(y_dev.data_ptr()),
                                    precision, ctypes.c_void_p(stream))
    assert rc == 0, lib().acg_last_error()
    torch.cuda.synchronize()
    return y_dev.cpu().numpy()


@pytest.mark.parametrize("precision,tol", [(0, TOL_FP64), (1, TOL_FP32)])
def test_matches_allocating_entry_two_calls_in_a_row(solver, precision, tol):
    rng = np.random.default_rng(3)
    for call in range(2):
        r = rng.standard_normal(solver.n)
        r -= r.mean()
        y_ref = solver.ldlsolve(r, "fp64" if precision == 0 else "mixed")
        y = _noalloc(solver, r, precision)
        assert np.all(np.isfinite(y))
        assert _rel(y, y_ref) < tol, (call, _rel(y, y_ref))


def test_rejects_graphs_above_the_limit(gpu_ok):
    import torch
    side = 400  # 160,000 vertices > ACG_NOALLOC_MAX_N = 131,072
    a = G.grid2(side)
    acgpu.seed(1)
    dev = acgpu.DeviceLapSolver(a, acgpu.approx_chol(a))
    r = torch.zeros(a.shape[0], dtype=torch.float64, device="cuda")
    y = torch.zeros_like(r)
    rc = lib().acg_ldlsolve_noalloc(dev._h, ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(y.data_ptr()), 0, None)
    assert rc == -1
    assert b"131072" in lib().acg_last_error()
    dev.close()
