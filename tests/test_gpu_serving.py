"""Serving: requests on several graphs arrive while others are running and
join each graph's device-resident serving loop as its slots free up.  Each
result must equal the same right-hand sides solved alone (FP64: x within
1e-7 after removing the mean, iterations within 1; mixed: true relative
residual <= tol and x within 1e-5 of the same right-hand side solved alone
in mixed precision); eviction under a tight HBM budget and rejection of a
graph larger than the budget are checked too."""
import threading
import time

import numpy as np
import pytest

import acgpu
from acgpu import generators as G
from acgpu.serving import AdmissionError, SolveServer
import oracle as O

pytestmark = pytest.mark.gpu


def _graphs():
    return {
        "g2": G.grid2(40, weights="loguniform", seed=1),
        "g3": G.grid3(14, weights="loguniform", seed=2),
        "pm": G.path_plus_matchings(3000, sigma=1.0, seed=3),
    }


def _rel(x, y):
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


def _submit_stream(server, graphs, nreq, seed):
    rng = np.random.default_rng(seed)
    names = sorted(graphs)
    futs = []

    def producer(tid):
        r = np.random.default_rng(seed + 100 + tid)
        for _ in range(nreq // 2):
            gid = names[r.integers(len(names))]
            n = graphs[gid].shape[0]
            k = int(r.integers(1, 6))
            B = r.standard_normal((n, k))
            futs.append((gid, B, server.submit(gid, B, tol=1e-9)))
            time.sleep(float(r.exponential(0.002)))

    ths = [threading.Thread(target=producer, args=(t,)) for t in range(2)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    return futs


def test_results_same_alone_and_in_the_mix(gpu_ok):
    graphs = _graphs()
    factors = {}
    for i, (gid, a) in enumerate(sorted(graphs.items())):
        acgpu.seed(10 + i)
        factors[gid] = acgpu.approx_chol(a)
    server = SolveServer(hbm_budget=8 << 30, slots=8, precision="fp64")
    for gid, a in graphs.items():
        server.register(gid, a, ldli=factors[gid])
    with server:
        futs = _submit_stream(server, graphs, 24, seed=5)
        results = [(gid, B, f.result(timeout=300)) for gid, B, f in futs]
    stats = server.latency_stats()
    assert stats["requests"] == len(futs) and stats["loop_launches"] < len(futs)
    alone = {gid: acgpu.DeviceLapSolver(graphs[gid], factors[gid]) for gid in graphs}
    for gid, B, (X, infos) in results:
        for c in range(B.shape[1]):
            its = [0]
            x1 = alone[gid](B[:, c], tol=1e-9, maxits=2000, pcgIts=its)
            assert abs(infos[c].iterations - its[0]) <= 1
            assert _rel(O.center(X[:, c]), O.center(x1)) < 1e-7
            assert O.relres(graphs[gid], X[:, c], B[:, c] - B[:, c].mean()) < 1e-8
    for s in alone.values():
        s.close()


def test_mixed_precision_serving_meets_tol(gpu_ok):
    graphs = _graphs()
    factors = {}
    for i, (gid, a) in enumerate(sorted(graphs.items())):
        acgpu.seed(20 + i)
        factors[gid] = acgpu.approx_chol(a)
    server = SolveServer(hbm_budget=8 << 30, slots=8, precision="mixed")
    for gid, a in graphs.items():
        server.register(gid, a, ldli=factors[gid])
    alone = {gid: acgpu.DeviceLapSolver(graphs[gid], factors[gid]) for gid in graphs}
    with server:
        futs = _submit_stream(server, graphs, 12, seed=9)
        for gid, B, f in futs:
            X, infos = f.result(timeout=300)
            for c in range(B.shape[1]):
                assert infos[c].status == 0
                assert O.relres(graphs[gid], X[:, c], B[:, c] - B[:, c].mean()) <= 1e-9 * 1.01
                x1 = alone[gid](B[:, c], tol=1e-9, maxits=2000, precision="mixed")
                assert _rel(O.center(X[:, c]), O.center(x1)) < 1e-5
    for s_ in alone.values():
        s_.close()


def test_admission_by_hbm_budget(gpu_ok):
    graphs = _graphs()
    one = max(SolveServer(0)._estimate_bytes(_entry(a)) for a in graphs.values())
    server = SolveServer(hbm_budget=one + 1, slots=8, precision="fp64")
    for i, (gid, a) in enumerate(sorted(graphs.items())):
        server.register(gid, a, seed=30 + i)
    with server:
        futs = [(gid, server.submit(gid, np.random.default_rng(j).standard_normal(graphs[gid].shape[0])))
                for j, gid in enumerate(["g2", "g3", "pm", "g2", "pm", "g3"])]
        for gid, f in futs:
            X, infos = f.result(timeout=300)
            assert infos[0].status == 0
    assert server._resident <= one + 1
    tiny = SolveServer(hbm_budget=1024, slots=8)
    tiny.register("g2", graphs["g2"], seed=1)
    with tiny:
        with pytest.raises(AdmissionError):
            tiny.submit("g2", np.ones(graphs["g2"].shape[0])).result(timeout=60)


def _entry(a):
    from acgpu.serving import _GraphEntry
    acgpu.seed(1)
    return _GraphEntry("x", a, acgpu.approx_chol(a))


def test_disconnected_graph_is_served_per_component(gpu_ok):
    """A disconnected graph: each component of at least 50 vertices is served
    by its own loop, smaller ones on the host, singletons get zero; the
    assembled x matches the exact solve of every component."""
    import scipy.sparse as sp
    parts = [G.grid2(12, weights="loguniform", seed=1), G.star_graph(9), G.path_plus_matchings(400, seed=2)]
    a = sp.block_diag(parts + [sp.csc_matrix((1, 1))] * 2, format="csc")
    a.sort_indices()
    n = a.shape[0]
    B = np.random.default_rng(3).standard_normal((n, 2))
    co = acgpu.components(a)
    for c in np.unique(co):
        m = co == c
        B[m] -= B[m].mean(axis=0)
    server = SolveServer(hbm_budget=8 << 30, slots=8, precision="fp64")
    server.register("u", a, seed=4)
    with server:
        X, infos = server.submit("u", B, tol=1e-10).result(timeout=300)
    assert server.latency_stats()["requests"] == 1
    for col in range(2):
        start = 0
        for p in parts:
            k = p.shape[0]
            xe = O.exact_solve(p, B[start:start + k, col])
            xs = X[start:start + k, col]
            assert np.linalg.norm((xs - xs.mean()) - xe) <= 1e-7 * np.linalg.norm(xe)
            start += k
        assert np.all(X[start:, col] == 0)
