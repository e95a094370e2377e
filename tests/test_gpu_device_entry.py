"""The device-pointer entry points (acg_solve_device, acg_solve_batch_device):
right-hand sides written on the legacy default stream (torch's default) are
read after that work, without a device-wide synchronization, and give the same
results as the host-buffer entry; a serving loop of another solver keeps
running meanwhile."""
import ctypes

import numpy as np
import pytest

import acgpu
import oracle as O
from acgpu import generators as G
from acgpu._lib import AcgSolveInfo, check, lib

pytestmark = pytest.mark.gpu


def test_device_entries_match_host_entry(gpu_ok):
    import torch
    a = G.grid3(16, weights="loguniform", seed=4)
    acgpu.seed(2)
    ldli = acgpu.approx_chol(a)
    n = a.shape[0]
    dev = acgpu.DeviceLapSolver(a, ldli)
    g2 = G.grid2(60, weights="loguniform", seed=5)
    other = acgpu.DeviceLapSolver(g2, acgpu.approx_chol(g2))
    loop = acgpu.ServeLoop(other, precision="mixed", slots=8)
    tickets = [loop.submit(np.random.default_rng(s).standard_normal(other.n), tol=1e-8) for s in range(12)]
    rng = np.random.default_rng(6)
    B = rng.standard_normal((5, n))
    # written on torch's (legacy) default stream just before the call
    Bd = torch.from_numpy(B).cuda() * 1.0
    Xd = torch.empty_like(Bd)
    info = (AcgSolveInfo * 5)()
    check(lib().acg_solve_device(dev._h, ctypes.c_void_p(Bd[0].data_ptr()), ctypes.c_void_p(Xd[0].data_ptr()), 1e-8,
                                 1000, float("inf"), 5, 0, info))
    x0 = dev(B[0], tol=1e-8, maxits=1000)
    assert np.allclose(Xd[0].cpu().numpy(), x0, rtol=0, atol=1e-12 * np.abs(x0).max())
    check(lib().acg_solve_batch_device(dev._h, ctypes.c_void_p(Bd.data_ptr()), ctypes.c_void_p(Xd.data_ptr()), 5, n,
                                       1e-8, 1000, float("inf"), 5, 1, info))
    X = Xd.cpu().numpy()
    for c in range(5):
        assert info[c].status == 0
        assert O.relres(a, X[c], B[c] - B[c].mean()) <= 1e-8 * 1.01
    for t in tickets:
        t.wait()
        assert t.info[0].status == 0
    loop.close()
    other.close()
    dev.close()
