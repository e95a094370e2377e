"""The device-resident serving loop (acg_serve_*): continuous batching.

Requests that arrive while others are on the GPU join the running loop as
slots free up (one loop launch serves them all), and each result is the same
request solved alone within the batched tests' tolerances:
  * FP64: iterations within 1 and x within 1e-7 (mean removed) of the same
    right-hand side solved alone;
  * mixed precision: true relres <= tol, and x within 1e-5 of the same right-
    hand side solved alone and of the exact (SuperLU) solution.
The reference solves one vector per call (src/approxChol.jl:1624).
"""
import threading
import time

import numpy as np
import pytest

import acgpu
import oracle as O
from acgpu import generators as G

pytestmark = pytest.mark.gpu


def _rel(x, y):
    x, y = O.center(x), O.center(y)
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


@pytest.fixture(scope="module")
def problem(gpu_ok):
    a = G.grid3(22, weights="loguniform", seed=9)
    acgpu.seed(3)
    return a, acgpu.approx_chol(a)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_requests_join_a_running_loop_and_match_alone(problem, precision):
    a, ldli = problem
    n = a.shape[0]
    dev = acgpu.DeviceLapSolver(a, ldli)
    rng = np.random.default_rng(11)
    blocks = [rng.standard_normal((n, int(k))) for k in rng.integers(1, 4, size=14)]
    tol = 1e-8
    loop = acgpu.ServeLoop(dev, precision=precision, slots=8, queue=40)
    tickets = [None] * len(blocks)
    # the first wave starts the loop; the rest arrive while it runs (a solve
    # here takes a millisecond or two, so the late ones follow at once)
    for i in range(4):
        tickets[i] = loop.submit(blocks[i], tol=tol)
    joined_while_running = 0

    def late():
        nonlocal joined_while_running
        for i in range(4, len(blocks)):
            if any(not tickets[j].done() for j in range(i)):
                joined_while_running += 1
            tickets[i] = loop.submit(blocks[i], tol=tol)
            time.sleep(0.0002)

    th = threading.Thread(target=late)
    th.start()
    th.join()
    results = [t.wait() for t in tickets]
    st = loop.stats()
    loop.close()
    assert st["completed"] == sum(b.shape[1] for b in blocks)
    assert joined_while_running > 0
    # the requests that arrived while the loop ran joined its launch
    assert st["launches"] < len(blocks)
    for blk, X, t in zip(blocks, results, tickets):
        for c in range(blk.shape[1]):
            b = blk[:, c]
            info = t.info[c]
            assert info.status == 0, info.status
            x1 = dev(b, tol=tol, maxits=2000, precision=precision)
            alone = dev.last_info[0]
            if precision == "fp64":
                assert abs(info.iterations - alone.iterations) <= 1, (info.iterations, alone.iterations)
                assert _rel(X[:, c], x1) < 1e-7
            else:
                assert O.relres(a, X[:, c], b - b.mean()) <= tol * 1.01
                assert _rel(X[:, c], x1) < 1e-5
                assert _rel(X[:, c], O.exact_solve(a, b)) < 1e-5
    dev.close()


def test_loop_edge_cases_and_relaunch(problem):
    a, ldli = problem
    n = a.shape[0]
    dev = acgpu.DeviceLapSolver(a, ldli)
    loop = acgpu.ServeLoop(dev, precision="fp64", slots=8)
    # zero right-hand side: x = 0 at once; maxits = 0: stops before any iteration
    t0 = loop.submit(np.zeros(n), tol=1e-8)
    x0 = t0.wait()
    assert np.all(x0 == 0) and t0.info[0].status == 0 and t0.info[0].iterations == 0
    t1 = loop.submit(np.random.default_rng(1).standard_normal(n), tol=1e-8, maxits=0)
    t1.wait()
    assert t1.info[0].status == 1 and t1.info[0].iterations == 0
    # a non-finite right-hand side is an input error; the loop goes on
    bad = np.random.default_rng(2).standard_normal(n)
    bad[5] = np.nan
    tb = loop.submit(bad, tol=1e-8)
    with pytest.raises(acgpu._lib.AcgError) as e:
        tb.wait()
    assert e.value.code == -1
    # the loop went idle between these requests and was relaunched each time
    b = np.random.default_rng(3).standard_normal(n)
    x = loop.submit(b, tol=1e-8).wait()
    assert O.relres(a, x, b - b.mean()) < 1e-7
    assert loop.stats()["launches"] >= 2
    # the batched entry points wait for the loop to close
    with pytest.raises(acgpu._lib.AcgError) as e:
        dev(np.random.default_rng(4).standard_normal((n, 4)), tol=1e-8)
    assert e.value.code == -6
    loop.close()
    dev(np.random.default_rng(4).standard_normal((n, 4)), tol=1e-8)
    dev.close()
