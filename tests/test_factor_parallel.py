"""The opt-in parallel elimination (acg_approxchol_parallel; not the
reference's): rounds of independent low-degree vertices eliminated at once
with the reference's per-vertex step (src/approxChol.jl:888-966) and keyed
random numbers.  Its factor is a different sample than approxChol's, so it is
checked for what it must be: a valid LDLinv (the same host checks acg_create
applies), independent of the thread count, and a preconditioner with which the
oracle's PCG (src/pcg.jl:256-445) converges about as fast as with the
reference's elimination."""
import ctypes

import numpy as np
import pytest

import acgpu
import oracle as O
from acgpu import generators as G
from acgpu._lib import lib


def _graphs():
    return {
        "grid2": G.grid2(60, weights="loguniform", seed=1),
        "grid3": G.grid3(18, weights="loguniform", seed=2),
        "matchings": G.path_plus_matchings(6000, sigma=2.0, seed=3),
        "rgg": G.largest_component(G.random_geometric(4000, seed=4)),
        "tree": G.random_tree(3000, seed=5),
        "star": G.star_graph(500),
    }


def _host_checks(a, f):
    h = ctypes.c_void_p()
    rc = lib().acg_create(a.shape[0], a.indptr.astype(np.int64), a.indices.astype(np.int64),
                          np.ascontiguousarray(a.data), f.col, f.colptr, f.rowval, f.fval, f.d, f.nnz, 1, None,
                          ctypes.byref(h))
    if rc == 0:
        lib().acg_destroy(h)
    return rc


@pytest.mark.parametrize("name", sorted(_graphs()))
def test_valid_thread_independent_and_converges(name):
    a = _graphs()[name]
    f1, r1 = acgpu.approx_chol_parallel(a, seed=7, threads=1)
    f4, r4 = acgpu.approx_chol_parallel(a, seed=7, threads=4)
    assert r1 == r4 >= 1
    for k in ("col", "colptr", "rowval", "fval", "d"):
        assert np.array_equal(getattr(f1, k), getattr(f4, k)), k
    assert f1.col.shape[0] == a.shape[0] - 1 and np.count_nonzero(f1.d == 0) == 1
    assert _host_checks(a, f1) in (0, -5)  # valid (-5: no device here, after the host checks)
    b = np.random.default_rng(1).standard_normal(a.shape[0])
    b -= b.mean()
    x, its, rc, _ = O.OracleSolver(a, f1)(b, tol=1e-8, maxits=500)
    assert rc == 0 and O.relres(a, x, b) < 1e-7
    acgpu.seed(7)
    _, its_ref, _, _ = O.OracleSolver(a, acgpu.approx_chol(a))(b, tol=1e-8, maxits=500)
    assert its <= 2 * its_ref + 5, (its, its_ref)


def test_seed_changes_the_sample():
    a = G.grid2(40, weights="loguniform", seed=1)
    f1, _ = acgpu.approx_chol_parallel(a, seed=1, threads=2)
    f2, _ = acgpu.approx_chol_parallel(a, seed=2, threads=2)
    assert not np.array_equal(f1.fval, f2.fval) or not np.array_equal(f1.rowval, f2.rowval)


def test_disconnected_graph_is_an_error():
    import scipy.sparse as sp
    a = sp.block_diag([G.grid2(5), G.grid2(4)], format="csc")
    a.sort_indices()
    with pytest.raises(acgpu._lib.AcgError):
        acgpu.approx_chol_parallel(a, seed=1, threads=2)
