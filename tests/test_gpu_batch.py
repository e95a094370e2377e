"""Batched right-hand sides through the C ABI: every column of a batch is its
own PCG system and must agree with the same right-hand side solved alone
(iteration counts within 1, x within 1e-7 after removing the mean for FP64;
true relative residual <= tol for mixed precision), and with the oracle."""
import numpy as np
import pytest

import acgpu
from acgpu import generators as G
import oracle as O

pytestmark = pytest.mark.gpu


def _rel(x, y):
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


@pytest.fixture(scope="module")
def grid(gpu_ok):
    a = G.grid3(16, weights="loguniform", seed=21)
    acgpu.seed(2)
    ldli = acgpu.approx_chol(a)
    dev = acgpu.DeviceLapSolver(a, ldli)
    yield a, ldli, dev
    dev.close()


@pytest.mark.parametrize("k", [5, 16, 40, 70])
def test_batch_matches_single_fp64(grid, k):
    a, ldli, dev = grid
    n = a.shape[0]
    B = np.random.default_rng(k).standard_normal((n, k))
    B[:, 1] = 0.0  # a zero right-hand side stops at set-up with x = 0
    X = dev(B, tol=1e-9, maxits=400)
    infos = list(dev.last_info)
    assert X.shape == (n, k)
    assert np.all(X[:, 1] == 0) and infos[1].iterations == 0
    for c in [0, 2, k - 1]:
        its = [0]
        x1 = dev(B[:, c], tol=1e-9, maxits=400, pcgIts=its)
        assert abs(infos[c].iterations - its[0]) <= 1, (c, infos[c].iterations, its[0])
        assert _rel(O.center(X[:, c]), O.center(x1)) < 1e-7
        assert O.relres(a, X[:, c], B[:, c] - B[:, c].mean()) < 1e-8


@pytest.mark.parametrize("k", [8, 33])
def test_batch_mixed_true_residual(grid, k):
    a, ldli, dev = grid
    n = a.shape[0]
    B = np.random.default_rng(100 + k).standard_normal((n, k))
    X = dev(B, tol=1e-8, maxits=2000, precision="mixed")
    for c in range(k):
        assert dev.last_info[c].status == 0
        assert O.relres(a, X[:, c], B[:, c] - B[:, c].mean()) <= 1e-8 * 1.01
    xe = O.exact_solve(a, B[:, 0])
    assert _rel(O.center(X[:, 0]), xe) < 1e-5


def test_batch_oracle_and_maxits(grid):
    a, ldli, dev = grid
    n = a.shape[0]
    orc = O.OracleSolver(a, ldli)
    B = np.random.default_rng(7).standard_normal((n, 12))
    X = dev(B, tol=1e-12, maxits=6)
    for c in range(12):
        assert dev.last_info[c].iterations == 6 and dev.last_info[c].status == 1
    xo, ito, rco, _ = orc(B[:, 3], tol=1e-12, maxits=6)
    assert ito == 6 and _rel(O.center(X[:, 3]), O.center(xo)) < 1e-8


def test_batch_repeatable(grid):
    a, ldli, dev = grid
    B = np.random.default_rng(9).standard_normal((a.shape[0], 24))
    X1 = dev(B, tol=1e-9)
    X2 = dev(B, tol=1e-9)
    assert np.array_equal(X1, X2)


def test_batch_stop_codes_on_the_tenth_iterations(grid):
    """The third L1 test, maxtime and maxits of every 10th iteration run after
    the p update (where |z|_1 is summed): maxits landing on those iterations
    stops every column there, and a tolerance no solve reaches ends every
    column with a stagnation code (src/pcg.jl:288-432), as a lone solve does."""
    a, ldli, dev = grid
    n = a.shape[0]
    B = np.random.default_rng(31).standard_normal((n, 8))
    for maxits in (10, 20):
        dev(B, tol=1e-14, maxits=maxits)
        for c in range(8):
            assert dev.last_info[c].iterations == maxits and dev.last_info[c].status == 1
    X = dev(B, tol=1e-30, maxits=400)
    infos = list(dev.last_info)
    stagnation = {2, 3, 4, 6}
    for c in range(8):
        assert infos[c].status in stagnation, (c, infos[c].status)
        assert O.relres(a, X[:, c], B[:, c] - B[:, c].mean()) < 1e-10
    its = [0]
    dev(B[:, 5], tol=1e-30, maxits=400, pcgIts=its)
    assert dev.last_info[0].status in stagnation
