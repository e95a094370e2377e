"""The serving layer's host logic (acgpu.serving.SolveServer) on the CPU, with
the device solver and its serving loop replaced by fakes: requests from two
producer threads on three graphs, a disconnected graph split into its
components, HBM-budget eviction, and a loop that fails.  Every future must
resolve; the GPU tests check the numbers."""
import threading
import time

import numpy as np
import pytest

import acgpu
import acgpu.serving as SV
from acgpu import generators as G


class _FakeSolver:
    def __init__(self, a, ldli, **kw):
        self.n = a.shape[0]

    def close(self):
        pass


class _FakeInfo:
    def __init__(self, its):
        self.iterations = its
        self.status = 0


class _FakeTicket:
    def __init__(self, B, fail):
        self._X = B * 2.0  # "solution": twice the right-hand side, so assembly is checkable
        self._fail = fail
        self._t_end = time.perf_counter() + float(np.random.default_rng().uniform(0.0005, 0.005))
        self.info = []

    def done(self):
        if self._fail and time.perf_counter() > self._t_end:
            raise RuntimeError("loop launch failed")
        return time.perf_counter() > self._t_end

    def wait(self):
        while time.perf_counter() <= self._t_end:
            time.sleep(0.0005)
        if self._fail:
            raise RuntimeError("loop launch failed")
        self.info = [_FakeInfo(7) for _ in range(self._X.shape[1])]
        return self._X


class _FakeLoop:
    fail_gid_n = None  # graphs of this many vertices fail

    def __init__(self, solver, precision, slots, queue):
        self.n = solver.n

    def submit(self, B, tol, maxits):
        return _FakeTicket(B, self.n == _FakeLoop.fail_gid_n)

    def stats(self):
        return {"launches": 1, "completed": 0}

    def close(self):
        pass


@pytest.fixture
def fakes(monkeypatch):
    monkeypatch.setattr(SV, "DeviceLapSolver", _FakeSolver)
    monkeypatch.setattr(SV, "ServeLoop", _FakeLoop)
    _FakeLoop.fail_gid_n = None
    yield


def _graphs():
    return {"g2": G.grid2(20, weights="loguniform", seed=1), "g3": G.grid3(8, weights="loguniform", seed=2),
            "pm": G.path_plus_matchings(600, sigma=1.0, seed=3)}


def _stream(server, graphs, nreq, seed):
    names = sorted(graphs)
    futs, lock = [], threading.Lock()

    def producer(tid):
        r = np.random.default_rng(seed + tid)
        for _ in range(nreq // 2):
            gid = names[r.integers(len(names))]
            B = r.standard_normal((graphs[gid].shape[0], int(r.integers(1, 4))))
            f = server.submit(gid, B, tol=1e-9)
            with lock:
                futs.append((gid, B, f))
            time.sleep(float(r.exponential(0.0005)))

    ths = [threading.Thread(target=producer, args=(t,)) for t in range(2)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    return futs


def test_every_request_resolves_and_is_assembled(fakes):
    graphs = _graphs()
    server = SV.SolveServer(hbm_budget=8 << 30, slots=8, precision="fp64")
    for gid, a in graphs.items():
        server.register(gid, a, seed=1)
    with server:
        futs = _stream(server, graphs, 40, seed=5)
        for gid, B, f in futs:
            X, infos = f.result(timeout=30)
            assert np.array_equal(X, 2.0 * B) and len(infos) == B.shape[1]
    st = server.latency_stats()
    assert st["requests"] == len(futs) and not server._pending


def test_disconnected_graph_and_eviction(fakes):
    graphs = _graphs()
    one = max(SV.SolveServer(0)._estimate_bytes(SV._GraphEntry("x", a, acgpu.approx_chol(a)))
              for a in graphs.values())
    server = SV.SolveServer(hbm_budget=one + 1, slots=8, precision="fp64")
    for gid, a in graphs.items():
        server.register(gid, a, seed=2)
    # a graph of two large components and an isolated vertex
    import scipy.sparse as sp
    g = sp.block_diag([graphs["g2"], graphs["pm"], sp.csc_matrix((1, 1))], format="csc")
    server.register("dis", g, seed=3)
    with server:
        futs = [(gid, server.submit(gid, np.ones((graphs[gid].shape[0] if gid != "dis" else g.shape[0], 2))))
                for gid in ["g2", "g3", "pm", "dis", "g2", "dis", "g3"]]
        for gid, f in futs:
            X, infos = f.result(timeout=30)
            if gid == "dis":
                assert np.all(X[-1] == 0) and np.all(X[:-1] == 2.0)
    assert server._resident <= one + 1


def test_a_failing_loop_fails_its_requests_only(fakes):
    graphs = _graphs()
    _FakeLoop.fail_gid_n = graphs["g3"].shape[0]
    server = SV.SolveServer(hbm_budget=8 << 30, slots=8, precision="fp64")
    for gid, a in graphs.items():
        server.register(gid, a, seed=1)
    with server:
        futs = [(gid, server.submit(gid, np.ones(graphs[gid].shape[0]))) for gid in ["g2", "g3", "pm", "g3", "g2"]]
        for gid, f in futs:
            if gid == "g3":
                with pytest.raises(RuntimeError):
                    f.result(timeout=30)
            else:
                f.result(timeout=30)
