"""Asynchronous solves (acg_solve_async / acg_poll / acg_wait): each request
returns what the synchronous acg_solve returns for the same block, bit for
bit (the same kernels in the same order on other buffers), whatever the slot,
the host memory kind of x (page-locked or pageable), the interleaving with
synchronous solves, and the solver's lifetime."""
import ctypes

import numpy as np
import pytest

import acgpu
from acgpu import generators as G
from acgpu._lib import AcgSolveInfo, lib
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grid(gpu_ok):
    a = G.grid3(14, weights="loguniform", seed=5)
    acgpu.seed(4)
    ldli = acgpu.approx_chol(a)
    dev = acgpu.DeviceLapSolver(a, ldli, tol=1e-8, maxits=500)
    yield a, ldli, dev
    dev.close()


def _rhs(n, k, seed):
    return np.random.default_rng(seed).standard_normal((n, k))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_async_equals_sync(grid, precision):
    a, _, dev = grid
    n = a.shape[0]
    blocks = [_rhs(n, k, 10 + k) for k in (5, 64, 12, 2)]
    sync = [dev(B, precision=precision) for B in blocks]
    sync_info = []
    for B in blocks:
        dev(B, precision=precision)
        sync_info.append([(i.iterations, i.status, i.true_relres) for i in dev.last_info])
    reqs = [dev.solve_async(B, precision=precision) for B in blocks]  # the third waits for the first
    for B, r, xs, si in zip(blocks, reqs, sync, sync_info):
        x = r.wait()
        assert r.rc == 0
        assert np.array_equal(x, xs)
        assert [(i.iterations, i.status, i.true_relres) for i in r.info] == si
    for c in range(blocks[1].shape[1]):
        b = blocks[1][:, c]
        assert O.relres(a, reqs[1].wait()[:, c], b - b.mean()) <= 1e-8 * 1.01
    # one column goes through the batched kernels too
    b = blocks[0][:, 0]
    r = dev.solve_async(b, precision=precision)
    x = r.wait()
    assert x.shape == b.shape and r.rc == 0
    assert O.relres(a, x, b - b.mean()) <= 1e-8 * 1.01


def test_async_pinned_output_and_poll(grid):
    import torch
    a, _, dev = grid
    n, k = a.shape[0], 32
    B = _rhs(n, k, 77)
    ref = dev(B, precision="mixed")
    hb = torch.empty((k, n), dtype=torch.float64, pin_memory=True)
    hx = torch.empty((k, n), dtype=torch.float64, pin_memory=True)
    hb.numpy()[:] = B.T
    L = lib()
    req = ctypes.c_void_p()
    rc = L.acg_solve_async(dev._h, hb.data_ptr(), hx.data_ptr(), k, n, 1e-8, 500, float("inf"), 5, 1,
                           ctypes.byref(req))
    assert rc == 0 and req.value
    seen = set()
    for _ in range(200000):
        p = L.acg_poll(req)
        assert p in (0, 1)
        seen.add(p)
        if p == 1:
            break
    assert 1 in seen
    infos = (AcgSolveInfo * k)()
    assert L.acg_wait(req, infos) == 0
    assert np.array_equal(hx.numpy().T, ref)
    assert all(i.status == 0 for i in infos)


def test_async_interleaves_with_sync_and_survives_destroy(grid):
    a, ldli, _ = grid
    n = a.shape[0]
    dev = acgpu.DeviceLapSolver(a, ldli, tol=1e-8, maxits=500)
    B1, B2, B3 = _rhs(n, 8, 1), _rhs(n, 8, 2), _rhs(n, 3, 3)
    ref1, ref2, ref3 = dev(B1), dev(B2), dev(B3)
    r1 = dev.solve_async(B1)
    x3 = dev(B3)  # a synchronous solve collects the open request first
    r2 = dev.solve_async(B2)
    assert np.array_equal(x3, ref3)
    dev.close()  # requests still open are finished and keep their results
    assert r1.done() and r2.done()
    assert np.array_equal(r1.wait(), ref1)
    assert np.array_equal(r2.wait(), ref2)


def test_async_bad_arguments(grid):
    a, _, dev = grid
    n = a.shape[0]
    L = lib()
    B = np.zeros((65, n))
    req = ctypes.c_void_p()
    assert L.acg_solve_async(dev._h, B.ctypes.data, B.ctypes.data, 65, n, 1e-8, 10, 1.0, 5, 0,
                             ctypes.byref(req)) == -1
    assert L.acg_solve_async(dev._h, B.ctypes.data, B.ctypes.data, 2, n - 1, 1e-8, 10, 1.0, 5, 0,
                             ctypes.byref(req)) == -1
    assert not req.value
    assert L.acg_poll(None) == -1 and L.acg_wait(None, None) == -1
