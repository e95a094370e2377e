"""Factors of the fixed elimination orders (:given, :wdeg, :random;
src/approxChol.jl:1628-1789) through the GPU solve: LDLsolver parity with the
oracle on the same factor (1e-12, FP64), and full solves to tolerance."""
import numpy as np
import pytest

import acgpu
from acgpu import generators as G
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", ["deg", "given", "wdeg", "random"])
def test_orderings_solve(gpu_ok, order):
    a = G.grid2(50, weights="loguniform", seed=9)
    params = acgpu.ApproxCholParams(order=order)
    acgpu.seed(4)
    ldli = acgpu.approx_chol(a, params)
    dev = acgpu.DeviceLapSolver(a, ldli, params=params)
    r = np.random.default_rng(1).standard_normal(a.shape[0])
    r -= r.mean()
    assert np.linalg.norm(dev.ldlsolve(r) - O.ldlsolve(ldli, r)) / np.linalg.norm(O.ldlsolve(ldli, r)) < 1e-12
    b = np.random.default_rng(2).standard_normal(a.shape[0])
    for prec in ("fp64", "mixed"):
        x = dev(b, tol=1e-8, maxits=3000, precision=prec)
        assert O.relres(a, x, b - b.mean()) <= 1e-8 * 1.01 if prec == "mixed" else \
            dev.last_info[0].status == 0
    st = dev.stats()
    assert st["levels"] >= 1 and st["nnz_factor"] == ldli.nnz
    dev.close()
    # the closure route with the same params
    acgpu.seed(4)
    f = acgpu.approxchol_lap(a, tol=1e-8, params=params, precision="mixed")
    x = f(b)
    assert O.relres(a, x, b - b.mean()) <= 1e-8 * 1.01


def test_approxchol_lap2(gpu_ok):
    """approxchol_lap2: the split/merge factor (src/approxChol.jl:1559-1578)
    through the same GPU solve."""
    a = G.grid3(14, weights="loguniform", seed=12)
    params = acgpu.ApproxCholParams("deg", 5, 2, 2)
    acgpu.seed(6)
    ldli = acgpu.approx_chol(a, params)
    dev = acgpu.DeviceLapSolver(a, ldli, params=params)
    r = np.random.default_rng(3).standard_normal(a.shape[0])
    r -= r.mean()
    y = O.ldlsolve(ldli, r)
    assert np.linalg.norm(dev.ldlsolve(r) - y) / np.linalg.norm(y) < 1e-12
    dev.close()
    b = np.random.default_rng(4).standard_normal(a.shape[0])
    acgpu.seed(6)
    f = acgpu.approxchol_lap2(a, tol=1e-8, precision="mixed")
    x = f(b)
    assert O.relres(a, x, b - b.mean()) <= 1e-8 * 1.01


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_parallel_factor_on_the_gpu(gpu_ok, precision):
    """The opt-in parallel elimination's factor (acg_approxchol_parallel) is an
    LDLinv like any other: the GPU solve with it agrees with the oracle's on
    the same factor, and its DAG is shallower than the :deg factor's."""
    a = G.grid3(24, weights="loguniform", seed=6)
    f, rounds = acgpu.approx_chol_parallel(a, seed=3, threads=4)
    acgpu.seed(3)
    fdeg = acgpu.approx_chol(a)
    dev = acgpu.DeviceLapSolver(a, f)
    ddeg = acgpu.DeviceLapSolver(a, fdeg)
    assert dev.stats()["levels"] < ddeg.stats()["levels"]
    ddeg.close()
    b = np.random.default_rng(4).standard_normal(a.shape[0])
    its = [0]
    x = dev(b, tol=1e-8, maxits=1000, pcgIts=its, precision=precision)
    xo, ito, _, _ = O.OracleSolver(a, f)(b, tol=1e-8, maxits=1000)
    if precision == "fp64":
        assert abs(its[0] - ito) <= 1
        assert np.linalg.norm(O.center(x) - O.center(xo)) <= 1e-7 * np.linalg.norm(O.center(xo))
    else:
        assert O.relres(a, x, b - b.mean()) <= 1e-8 * 1.01
    dev.close()
