"""The dense tail: the final levels of the LDLinv DAG applied as one dense
triangular product instead of level-by-level substitution.

It is the same linear operator as src/approxChol.jl:1347-1408 up to rounding,
so the FP64 LDLsolver must agree with the oracle to 1e-12 relative (the
tolerance of the sweep parity tests), with the same solver built without a
dense tail to 1e-12, and FP32 to 1e-4.  Tail sizes that do not fill the
32-row and 256-index tiles of the dense kernels are covered, as are the
batched (several right-hand sides) path and full PCG solves.
"""
import numpy as np
import pytest

import acgpu
from acgpu import generators as G
import oracle as O

pytestmark = pytest.mark.gpu


def _rel(x, y):
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


GRAPHS = [
    ("grid3_20_logw", lambda: G.grid3(20, weights="loguniform", seed=31)),
    ("grid2_90", lambda: G.grid2(90)),
    ("pm_12000", lambda: G.path_plus_matchings(12000, seed=32)),
]


@pytest.fixture(scope="module", params=GRAPHS, ids=[g[0] for g in GRAPHS])
def graph(gpu_ok, request):
    a = request.param[1]()
    acgpu.seed(3)
    ldli = acgpu.approx_chol(a)
    plain = acgpu.DeviceLapSolver(a, ldli, options=dict(dense_tail=-1))
    yield a, ldli, plain
    plain.close()


@pytest.mark.parametrize("kmax", [0, 1000, 777, 33])
def test_ldlsolve_with_dense_tail(graph, kmax):
    a, ldli, plain = graph
    n = a.shape[0]
    dev = acgpu.DeviceLapSolver(a, ldli, options=dict(dense_tail=kmax))
    st = dev.stats()
    assert plain.stats()["dense_vertices"] == 0
    limit = min(kmax if kmax > 0 else 4096, n // 4)
    assert 0 <= st["dense_vertices"] <= limit
    if kmax in (0, 1000):
        assert st["dense_vertices"] > 0 and st["dense_levels"] >= 8
    rng = np.random.default_rng(kmax)
    r = rng.standard_normal(n)
    r -= r.mean()
    y_ref = O.ldlsolve(ldli, r)
    y = dev.ldlsolve(r)
    assert _rel(y, y_ref) < 1e-12
    assert _rel(y, plain.ldlsolve(r)) < 1e-12
    assert _rel(dev.ldlsolve(r, "mixed"), y_ref) < 1e-4
    # twice in a row: the dense step keeps no state between calls
    assert np.array_equal(dev.ldlsolve(r), y)
    dev.close()


def test_solves_with_dense_tail(graph):
    a, ldli, plain = graph
    n = a.shape[0]
    dev = acgpu.DeviceLapSolver(a, ldli)
    assert dev.stats()["dense_vertices"] > 0
    orc = O.OracleSolver(a, ldli)
    b = np.random.default_rng(5).standard_normal(n)
    its = [0]
    x = dev(b, tol=1e-9, maxits=500, pcgIts=its)
    xo, ito, _, _ = orc(b, tol=1e-9, maxits=500)
    assert abs(its[0] - ito) <= 1
    assert _rel(O.center(x), O.center(xo)) < 1e-7
    xm = dev(b, tol=1e-8, maxits=2000, precision="mixed")
    assert O.relres(a, xm, b - b.mean()) <= 1e-8 * 1.01
    # batched columns through the dense tail agree with the solver without one
    B = np.random.default_rng(6).standard_normal((n, 12))
    X = dev(B, tol=1e-9, maxits=500)
    Xp = plain(B, tol=1e-9, maxits=500)
    for c in range(12):
        assert _rel(O.center(X[:, c]), O.center(Xp[:, c])) < 1e-7
    Xm = dev(B, tol=1e-8, maxits=2000, precision="mixed")
    for c in range(12):
        assert O.relres(a, Xm[:, c], B[:, c] - B[:, c].mean()) <= 1e-8 * 1.01
    dev.close()


def test_kernel_timing_with_dense_tail(graph):
    """The timing entry points run every sweep variant (with and without the
    dense products) to completion: no wait gives up."""
    a, ldli, plain = graph
    dev = acgpu.DeviceLapSolver(a, ldli)
    for prec in ("fp64", "mixed"):
        kt = dev.time_kernels(prec, reps=2)
        assert kt["dense_ms"] > 0 and kt["forward_sweep_ms"] > 0 and kt["backward_sweep_ms"] > 0
        assert kt["launches_per_iteration"] == 12 and kt["forward_launches"] == 3
        kb = dev.time_kernels_batch(16, prec, reps=2)
        assert kb["dense_ms"] > 0 and kb["forward_sweep_ms"] > 0 and kb["backward_sweep_ms"] > 0
        # batched loop body: mat-vec, pq, update, 2 sweeps, kb_yzr, kb_pupdate_z, 4 dense
        assert kb["launches_per_iteration"] == 11
    # the solver still solves correctly afterwards
    b = np.random.default_rng(8).standard_normal(a.shape[0])
    x = dev(b, tol=1e-8, maxits=2000, precision="mixed")
    assert O.relres(a, x, b - b.mean()) <= 1e-8 * 1.01
    kp = plain.time_kernels("fp64", reps=2)
    assert kp["dense_ms"] == 0 and kp["launches_per_iteration"] == 8
    dev.close()


def test_sweep_levels_timing(graph):
    """acg_time_sweep_levels: the forward prefixes grow and the backward
    suffixes shrink with the level; the deepest swept level leaves the backward
    sweep its own tasks only, and levels past the end are clamped."""
    a, ldli, plain = graph
    for solver in (acgpu.DeviceLapSolver(a, ldli), plain):
        st = solver.stats()
        swept = st["levels"] - st["dense_levels"]
        pts = [0, 1, swept // 2, swept - 1, st["levels"] + 10]
        for prec in ("fp64", "mixed"):
            rows = solver.time_sweep_levels(pts, nrhs=16, precision=prec, reps=2)
            ft = [r["forward_tasks"] for r in rows]
            bt = [r["backward_tasks"] for r in rows]
            assert all(0 < x <= y for x, y in zip(ft, ft[1:]))
            assert all(x >= y for x, y in zip(bt, bt[1:]))
            assert bt[0] > bt[3] > 0
            # the last level is swept only without a dense tail
            assert bt[-1] == (bt[3] if st["dense_levels"] == 0 else 0)
            # differences of timings: tiny prefixes may be within the noise (reported as 0)
            assert all(r["forward_ms"] >= 0 and r["backward_ms"] >= 0 for r in rows)
            assert rows[-1]["forward_ms"] > 0 and rows[0]["backward_ms"] > 0
        # still solves correctly afterwards
        b = np.random.default_rng(9).standard_normal(a.shape[0])
        x = solver(b, tol=1e-8, maxits=2000, precision="mixed")
        assert O.relres(a, x, b - b.mean()) <= 1e-8 * 1.01
        if solver is not plain:
            solver.close()
