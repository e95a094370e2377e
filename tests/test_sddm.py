"""approxchol_sddm: the reference's sddmWrapLap(approxchol_lap)
(src/solverInterface.jl:324-350, src/graphOps.jl:43-79).  The grounding step
is checked on the CPU (the extended graph's Laplacian restricted to the
original vertices is the SDDM matrix); solves run on the GPU."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import acgpu
from acgpu import generators as G
from acgpu.solvers import adj_val_and_excess, extend_matrix, lap


def _sddm(n_side=30, frac=0.1, seed=0):
    a = G.grid2(n_side, weights="loguniform", seed=seed)
    rng = np.random.default_rng(seed)
    extra = np.where(rng.random(a.shape[0]) < frac, rng.uniform(0.01, 1.0, a.shape[0]), 0.0)
    return sp.csc_matrix(lap(a) + sp.diags(extra)), a, extra


def test_grounding_reproduces_the_matrix():
    m, a, extra = _sddm()
    a0, dval, dexcess = adj_val_and_excess(m)
    assert abs(a0 - a).max() < 1e-15
    assert np.allclose(dexcess, extra, atol=1e-12)
    a1 = extend_matrix(a0, dval, dexcess)
    n = m.shape[0]
    assert a1.shape == (n + 1, n + 1)
    assert (a1.diagonal() == 0).all()
    l1 = lap(a1)
    assert abs(l1[:n, :n] - m).max() < 1e-12
    # no excess: no extension
    a2 = extend_matrix(a0, dval, np.zeros(n))
    assert a2.shape == (n, n)


@pytest.mark.gpu
def test_sddm_solve_on_device(gpu_ok):
    m, a, extra = _sddm(40, frac=0.05, seed=3)
    b = np.random.default_rng(1).standard_normal(m.shape[0])
    acgpu.seed(2)
    f = acgpu.approxchol_sddm(m, tol=1e-10, maxits=500)
    x = f(b)
    xe = spla.spsolve(m, b)
    assert np.linalg.norm(m @ x - b) / np.linalg.norm(b) < 1e-8
    assert np.linalg.norm(x - xe) / np.linalg.norm(xe) < 1e-6
    x2 = f(b, tol=1e-4)  # per-call tolerance, as the reference closure takes
    assert np.linalg.norm(m @ x2 - b) / np.linalg.norm(b) < 1e-2


@pytest.mark.gpu
def test_sddm_without_excess_is_a_laplacian_solve(gpu_ok):
    a = G.grid2(20)
    m = sp.csc_matrix(lap(a))
    b = np.random.default_rng(4).standard_normal(m.shape[0])
    b -= b.mean()
    acgpu.seed(2)
    x = acgpu.approxchol_sddm(m, tol=1e-9)(b)
    assert np.linalg.norm(m @ x - b) / np.linalg.norm(b) < 1e-7
