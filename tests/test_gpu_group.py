"""Many graphs in one launch: every graph of a group is its own PCG system and
must agree with the same graph solved alone (iterations within 1, x within
1e-7 after removing the mean) and with the oracle; graphs stop independently
(a tree in 1-2 iterations, grids in tens), a zero right-hand side stops at
set-up, and repeated solves are bitwise identical."""
import numpy as np
import pytest

import acgpu
from acgpu import generators as G
import oracle as O

pytestmark = pytest.mark.gpu


def _rel(x, y):
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


@pytest.fixture(scope="module")
def group(gpu_ok):
    graphs = [G.grid2(20 + 7 * i, weights="loguniform", seed=i) for i in range(4)]
    graphs += [G.largest_component(G.random_geometric(800 + 300 * i, seed=10 + i)) for i in range(4)]
    graphs += [G.random_tree(500, seed=3), G.path_plus_matchings(1200, seed=4), G.grid3(9, weights="loguniform", seed=5),
               G.cycle_graph(300, np.linspace(0.2, 2, 300))]
    factors = []
    for i, a in enumerate(graphs):
        acgpu.seed(100 + i)
        factors.append(acgpu.approx_chol(a))
    gs = acgpu.GroupSolver(graphs, factors)
    yield graphs, factors, gs
    gs.close()


def test_group_matches_each_graph_alone(group):
    graphs, factors, gs = group
    rng = np.random.default_rng(1)
    bs = [rng.standard_normal(a.shape[0]) for a in graphs]
    bs[5] = np.zeros(graphs[5].shape[0])
    xs = gs(bs, tol=1e-9, maxits=500)
    infos = gs.last_info
    assert infos[5].iterations == 0 and np.all(xs[5] == 0)
    assert infos[8].iterations <= 2  # the tree: exact factor
    for g, (a, f) in enumerate(zip(graphs, factors)):
        if g == 5:
            continue
        dev = acgpu.DeviceLapSolver(a, f)
        its = [0]
        x1 = dev(bs[g], tol=1e-9, maxits=500, pcgIts=its)
        dev.close()
        assert abs(infos[g].iterations - its[0]) <= 1, (g, infos[g].iterations, its[0])
        assert _rel(O.center(xs[g]), O.center(x1)) < 1e-7
        assert O.relres(a, xs[g], bs[g] - bs[g].mean()) < 1e-8
    orc = O.OracleSolver(graphs[0], factors[0])
    xo, ito, _, _ = orc(bs[0], tol=1e-9, maxits=500)
    assert abs(ito - infos[0].iterations) <= 1 and _rel(O.center(xs[0]), O.center(xo)) < 1e-7


def test_group_repeatable_and_reusable(group):
    graphs, factors, gs = group
    rng = np.random.default_rng(2)
    bs = [rng.standard_normal(a.shape[0]) for a in graphs]
    x1 = gs(bs, tol=1e-8)
    x2 = gs(bs, tol=1e-8)
    for a, b in zip(x1, x2):
        assert np.array_equal(a, b)
    gs(bs, tol=1e-12, maxits=4)  # a stop by maxits, except where the factor is exact
    for g, info in enumerate(gs.last_info):
        if g in (8, 11):  # tree and cycle: exact factors converge at once even at tol 1e-12
            assert info.status == 0 and info.iterations <= 2
        else:
            assert info.iterations == 4 and info.status == 1, (g, info.iterations, info.status)


def test_group_mixed_precision_matches_each_graph_alone(group):
    """Each graph's FP32 PCG inside its own FP64 refinement, all graphs in the
    same launches: every graph reaches the true residual tolerance and agrees
    with the same graph solved alone in mixed precision (x within 1e-6 of it,
    mean removed) and with the exact solution."""
    graphs, factors, gs = group
    rng = np.random.default_rng(5)
    bs = [rng.standard_normal(a.shape[0]) for a in graphs]
    bs[5] = np.zeros(graphs[5].shape[0])
    xs = gs(bs, tol=1e-9, maxits=2000, precision="mixed")
    infos = gs.last_info
    assert infos[5].status == 0 and np.all(xs[5] == 0)
    for g, (a, f) in enumerate(zip(graphs, factors)):
        if g == 5:
            continue
        b = bs[g] - bs[g].mean()
        assert infos[g].status == 0, (g, infos[g].status)
        assert O.relres(a, xs[g], b) <= 1e-9 * 1.01, (g, O.relres(a, xs[g], b))
        assert infos[g].true_relres <= 1e-9 * 1.01
        dev = acgpu.DeviceLapSolver(a, f)
        x1 = dev(bs[g], tol=1e-9, maxits=2000, precision="mixed")
        dev.close()
        assert _rel(O.center(xs[g]), O.center(x1)) < 1e-6, g
        xe = O.exact_solve(a, bs[g])
        assert _rel(O.center(xs[g]), xe) < 1e-5, g
    # repeatable
    xs2 = gs(bs, tol=1e-9, maxits=2000, precision="mixed")
    for a1, a2 in zip(xs, xs2):
        assert np.array_equal(a1, a2)
