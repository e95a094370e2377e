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


# The sweep layouts acg_ldlsolve_noalloc branches on: the default sync-free
# sweep with its dense tail, the per-level engine, the one-CTA tail engine, no
# dense tail, and one value per vertex in the ordinary entry's vectors.
LAYOUTS = {
    "default": {},
    "per_level": dict(sweep_lanes=1),
    "one_cta_tail": dict(sweep_lanes=1, tail=2),
    "no_dense_tail": dict(dense_tail=-1),
    "packed": dict(sweep_stride=1),
}


@pytest.fixture(scope="module", params=sorted(LAYOUTS))
def solver(gpu_ok, request):
    a = G.grid3(18, weights="loguniform", seed=11)
    acgpu.seed(5)
    dev = acgpu.DeviceLapSolver(a, acgpu.approx_chol(a), options=LAYOUTS[request.param])
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
    import torch
    rng = np.random.default_rng(3)
    for call in range(2):
        r = rng.standard_normal(solver.n)
        r -= r.mean()
        y_ref = solver.ldlsolve(r, "fp64" if precision == 0 else "mixed")
        r_dev = torch.from_numpy(r).to("cuda")
        y_dev = torch.full_like(r_dev, float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib().acg_ldlsolve_noalloc(solver._h, ctypes.c_void_p(r_dev.data_ptr()),
                                        ctypes.c_void_p(y_dev.data_ptr()), precision,
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, lib().acg_last_error()
        torch.cuda.synchronize()
        # nothing was allocated on the device by the call
        assert torch.cuda.mem_get_info()[0] == free_before
        y = y_dev.cpu().numpy()
        assert np.all(np.isfinite(y))
        assert _rel(y, y_ref) < tol, (call, _rel(y, y_ref))


def test_rejects_a_group_solver(gpu_ok):
    import torch
    graphs = [G.grid2(12, weights="loguniform", seed=s) for s in (1, 2)]
    acgpu.seed(2)
    grp = acgpu.GroupSolver(graphs, [acgpu.approx_chol(g) for g in graphs])
    r = torch.zeros(grp.n, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(r)
    rc = lib().acg_ldlsolve_noalloc(grp._h, ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(y.data_ptr()), 0, None)
    assert rc == -1
    assert b"group" in lib().acg_last_error()
    grp.close()


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
