"""approxchol_lap on a disconnected graph follows lapWrapComponents
(src/solverInterface.jl:212-275): singletons get zero, components with fewer
than 50 vertices a direct solve, larger ones the GPU solver, all of the large
ones together in one group launch; x agrees with the exact solution per
component, and pcgIts is the largest count over components."""
import numpy as np
import pytest
import scipy.sparse as sp

import acgpu
from acgpu import generators as G
import oracle as O

pytestmark = pytest.mark.gpu


def _union(parts, isolated):
    blocks = list(parts) + [sp.csc_matrix((1, 1))] * isolated
    a = sp.block_diag(blocks, format="csc")
    a.sort_indices()
    return a


def test_components_match_exact(gpu_ok):
    parts = [G.grid2(12, weights="loguniform", seed=1), G.cycle_graph(20, np.linspace(0.5, 2, 20)),
             G.path_plus_matchings(300, seed=2), G.star_graph(7)]
    a = _union(parts, 5)
    n = a.shape[0]
    rng = np.random.default_rng(0)
    b = rng.standard_normal(n)
    # make b orthogonal to every component's constant vector (the solvable part)
    co = acgpu.components(a)
    for c in np.unique(co):
        m = co == c
        b[m] -= b[m].mean()
    acgpu.seed(3)
    its = [0]
    f = acgpu.approxchol_lap(a, tol=1e-10, pcgIts=its)
    x = f(b)
    start = 0
    for p in parts:
        k = p.shape[0]
        xe = O.exact_solve(p, b[start:start + k])
        xs = x[start:start + k]
        assert np.linalg.norm((xs - xs.mean()) - xe) <= 1e-7 * max(np.linalg.norm(xe), 1e-30)
        start += k
    assert np.all(x[start:] == 0)  # singletons
    assert its[0] >= 1
    la = acgpu.lap(a)
    assert np.linalg.norm(la @ x - b) / np.linalg.norm(b) < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_components_share_one_group_launch(gpu_ok, precision):
    """Singletons, small components and four large ones: the large ones are one
    GroupSolver (one launch per right-hand side), each agreeing with its exact
    solve; several right-hand sides at once work column by column."""
    parts = [G.grid2(15, weights="loguniform", seed=1), G.star_graph(9),
             G.path_plus_matchings(400, seed=2), G.grid3(8, weights="loguniform", seed=3),
             G.cycle_graph(30, np.linspace(0.5, 2, 30)), G.largest_component(G.random_geometric(900, seed=4))]
    a = _union(parts, 3)
    n = a.shape[0]
    co = acgpu.components(a)
    B = np.random.default_rng(1).standard_normal((n, 3))
    for c in np.unique(co):
        m = co == c
        B[m] -= B[m].mean(axis=0)
    acgpu.seed(8)
    its = [0]
    f = acgpu.approxchol_lap(a, tol=1e-10, pcgIts=its, precision=precision)
    assert f.group is not None and f.group.group.ngraphs == 4
    X = f(B)
    assert its[0] >= 1
    for col in range(3):
        start = 0
        for p in parts:
            k = p.shape[0]
            xe = O.exact_solve(p, B[start:start + k, col])
            xs = X[start:start + k, col]
            assert np.linalg.norm((xs - xs.mean()) - xe) <= 1e-7 * max(np.linalg.norm(xe), 1e-30)
            start += k
        assert np.all(X[start:, col] == 0)


def test_negative_weight_error(gpu_ok):
    a = G.grid2(6).tolil()
    a[0, 1] = a[1, 0] = -2.0
    with pytest.raises(ValueError):
        acgpu.approxchol_lap(a.tocsc())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_one_large_component_with_isolated_vertices(gpu_ok, precision):
    """The common disconnected case: one component of at least 50 vertices plus
    a small one and isolated vertices.  The large one runs on the one-graph
    solver; a one-graph group solves too (as acg_solve does)."""
    big = G.grid2(30, weights="loguniform", seed=7)
    a = _union([big, G.path_graph(6)], 4)
    n = a.shape[0]
    co = acgpu.components(a)
    b = np.random.default_rng(2).standard_normal(n)
    for c in np.unique(co):
        b[co == c] -= b[co == c].mean()
    acgpu.seed(4)
    its = [0]
    f = acgpu.approxchol_lap(a, tol=1e-9, pcgIts=its, precision=precision)
    assert f.group is not None and f.group.group is None and f.group.single is not None
    x = f(b)
    assert O.relres(a, x, b) < 1e-8 and its[0] > 0
    assert np.all(x[-4:] == 0)
    acgpu.seed(4)
    ldli = acgpu.approx_chol(big)
    g1 = acgpu.GroupSolver([big], [ldli])
    nb = big.shape[0]
    xg = g1([b[:nb]], tol=1e-9, precision=precision)[0]
    assert O.relres(big, xg, b[:nb]) < 1e-8 and g1.last_info[0].status == 0
    g1.close()
