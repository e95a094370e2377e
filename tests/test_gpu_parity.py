"""GPU parity against the CPU oracle (restatement of the reference's solve
phase) on the same LDLinv, through the C ABI.

Tolerances (FP64 path): mat-vec and LDLsolver 1e-12 relative (the device folds
the running products of forward!/backward! into per-entry constants and sums
in a different order, so agreement is to rounding, not bitwise); PCG x within
1e-7 relative after removing the mean, iteration counts within 1.
FP32 preconditioner: 1e-4 relative.  Mixed solves: true relative residual <= tol.
"""
import math

import numpy as np
import pytest

import acgpu
from acgpu import generators as G
import oracle as O

pytestmark = pytest.mark.gpu


def _setup(a, seed=1):
    acgpu.seed(seed)
    ldli = acgpu.approx_chol(a)
    dev = acgpu.DeviceLapSolver(a, ldli)
    orc = O.OracleSolver(a, ldli)
    return ldli, dev, orc


def _rel(x, y):
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


GRAPHS = [
    ("grid2_60", lambda: G.grid2(60)),
    ("grid2_40_logw", lambda: G.grid2(40, weights="loguniform", seed=2)),
    ("grid3_14_logw", lambda: G.grid3(14, weights="loguniform", seed=3)),
    ("pm_5000", lambda: G.path_plus_matchings(5000, seed=4)),
    ("tree_3000", lambda: G.random_tree(3000, seed=5)),
    ("cycle_500", lambda: G.cycle_graph(500, np.linspace(0.1, 3, 500))),
    ("path_2", lambda: G.path_graph(2)),
    ("star_300", lambda: G.star_graph(300)),
]


@pytest.mark.parametrize("name,make", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_lap_mul_and_ldlsolve(gpu_ok, name, make):
    a = make()
    ldli, dev, orc = _setup(a)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(a.shape[0])
    assert _rel(dev.lap_mul(x), orc.lap.mul(x)) < 1e-12
    assert _rel(dev.lap_mul(x, "mixed"), orc.lap.mul(x)) < 1e-5
    r = x - x.mean()
    y_ref = O.ldlsolve(ldli, r)
    assert _rel(dev.ldlsolve(r), y_ref) < 1e-12
    assert _rel(dev.ldlsolve(r, "mixed"), y_ref) < 1e-4


@pytest.mark.parametrize("name,make", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_pcg_fp64_matches_oracle(gpu_ok, name, make):
    a = make()
    ldli, dev, orc = _setup(a, seed=3)
    b = np.random.default_rng(1).standard_normal(a.shape[0])
    its = [0]
    x = dev(b, tol=1e-8, maxits=500, pcgIts=its)
    xo, ito, rco, nro = orc(b, tol=1e-8, maxits=500)
    assert abs(its[0] - ito) <= 1, (its[0], ito)
    assert _rel(O.center(x), O.center(xo)) < 1e-7
    info = dev.last_info[0]
    assert info.status == rco or abs(its[0] - ito) == 1
    assert O.relres(a, x, b - b.mean()) < 1e-7


def test_grid2_200_fp64(gpu_ok):
    """grid2(200), one Gaussian RHS, tol 1e-6: GPU vs CPU on the same LDLinv."""
    a = G.grid2(200)
    ldli, dev, orc = _setup(a, seed=1)
    b = np.random.default_rng(7).standard_normal(a.shape[0])
    b -= b.mean()
    its = [0]
    x = dev(b, tol=1e-6, pcgIts=its)
    xo, ito, _, _ = orc(b, tol=1e-6)
    assert abs(its[0] - ito) <= 1
    assert _rel(O.center(x), O.center(xo)) < 1e-7
    assert O.relres(a, x, b) < 1e-6 * 1.01
    xe = O.exact_solve(a, b)
    assert _rel(O.center(x), xe) < 1e-3


@pytest.mark.parametrize("name,make", GRAPHS[:5], ids=[g[0] for g in GRAPHS[:5]])
def test_mixed_reaches_true_residual(gpu_ok, name, make):
    a = make()
    ldli, dev, orc = _setup(a, seed=5)
    b = np.random.default_rng(2).standard_normal(a.shape[0])
    b -= b.mean()
    x = dev(b, tol=1e-8, maxits=2000, precision="mixed")
    info = dev.last_info[0]
    assert info.status == 0, info.status
    assert O.relres(a, x, b) <= 1e-8 * 1.01
    assert info.true_relres <= 1e-8
    xe = O.exact_solve(a, b)
    assert _rel(O.center(x), xe) < 1e-5


def test_tree_factor_is_exact(gpu_ok):
    """On a tree every elimination is exact, so LDLsolver is the pseudo-inverse."""
    a = G.random_tree(2000, seed=9)
    ldli, dev, orc = _setup(a)
    b = np.random.default_rng(3).standard_normal(2000)
    b -= b.mean()
    xe = O.exact_solve(a, b)
    assert _rel(dev.ldlsolve(b), xe) < 1e-10
    its = [0]
    dev(b, tol=1e-10, pcgIts=its)
    assert its[0] <= 2


def test_stop_rules_and_edge_inputs(gpu_ok):
    a = G.grid2(50, weights="loguniform", seed=1)
    ldli, dev, orc = _setup(a)
    n = a.shape[0]
    b = np.random.default_rng(4).standard_normal(n)
    its = [0]
    dev(b, tol=1e-12, maxits=3, pcgIts=its)
    assert its[0] == 3 and dev.last_info[0].status == 1
    x = dev(b, maxits=0, pcgIts=its)
    assert its[0] == 0 and np.all(x == 0)
    x = dev(np.zeros(n), pcgIts=its)
    assert np.all(x == 0) and its[0] == 0
    x = dev(np.full(n, 3.0))  # mean removal leaves a zero rhs
    assert np.all(x == 0)
    # maxtime: stops after the first iteration that exceeds it
    x = dev(b, tol=1e-14, maxits=10 ** 6, maxtime=0.0, pcgIts=its)
    assert its[0] == 1 and dev.last_info[0].status == 7
    # same stop as the oracle on a maxits-limited run
    xo, ito, rco, _ = orc(b, tol=1e-12, maxits=7)
    x = dev(b, tol=1e-12, maxits=7, pcgIts=its)
    assert its[0] == ito == 7 and rco == 1
    assert _rel(O.center(x), O.center(xo)) < 1e-9


def test_repeatable_bitwise(gpu_ok):
    a = G.grid3(12, weights="loguniform", seed=8)
    ldli, dev, orc = _setup(a)
    b = np.random.default_rng(5).standard_normal(a.shape[0])
    x1 = dev(b, tol=1e-9)
    x2 = dev(b, tol=1e-9)
    assert np.array_equal(x1, x2)
    m1 = dev(b, tol=1e-9, precision="mixed")
    m2 = dev(b, tol=1e-9, precision="mixed")
    assert np.array_equal(m1, m2)


@pytest.mark.parametrize("name,make", GRAPHS[:5], ids=[g[0] for g in GRAPHS[:5]])
def test_sweep_vector_layout_is_invisible(gpu_ok, name, make):
    """One 32-byte sector per vertex in the sweep vectors (the default) and one
    value per vertex (sweep_stride=1) run the same arithmetic in the same
    order: LDLsolver and whole solves agree bit for bit."""
    a = make()
    acgpu.seed(1)
    ldli = acgpu.approx_chol(a)
    dev = acgpu.DeviceLapSolver(a, ldli)
    compact = acgpu.DeviceLapSolver(a, ldli, options=dict(sweep_stride=1))
    rng = np.random.default_rng(3)
    r = rng.standard_normal(a.shape[0])
    r -= r.mean()
    for prec in ("fp64", "mixed"):
        assert np.array_equal(dev.ldlsolve(r, prec), compact.ldlsolve(r, prec))
        assert np.array_equal(dev(r, tol=1e-9, maxits=300, precision=prec),
                              compact(r, tol=1e-9, maxits=300, precision=prec))
    dev.close()
    compact.close()
