"""Failure handling on the GPU, in the forms that neither fault nor hang it.

* A bounded sweep wait runs out.  The option test_unproduced_task blanks one
  record of the forward sweep tables, so the values of its vertices are never
  produced (a flag that nothing sets); with a short spin_limit the waits on
  them give up within milliseconds, the sweep raises its error flag, and every
  solve path returns ACG_ERR_TIMEOUT.  The context stays usable: a fresh
  solver on the same graph then solves normally.
* A right-hand side with a NaN or infinite entry is reported as
  ACG_ERR_INVALID by every solve path (the reference's pcg would iterate on
  NaNs until maxits, src/pcg.jl:256-445).
"""
import ctypes

import numpy as np
import pytest

import acgpu
import oracle as O
from acgpu import generators as G
from acgpu._lib import AcgError

pytestmark = pytest.mark.gpu

SHORT = dict(spin_limit=1 << 14, test_unproduced_task=1)


@pytest.fixture(scope="module")
def problem(gpu_ok):
    a = G.grid3(20, weights="loguniform", seed=5)
    acgpu.seed(2)
    return a, acgpu.approx_chol(a)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("k", [1, 16])
def test_a_wait_that_runs_out_is_reported_and_the_context_survives(problem, precision, k):
    a, ldli = problem
    n = a.shape[0]
    B = np.random.default_rng(1).standard_normal((n, k))
    bad = acgpu.DeviceLapSolver(a, ldli, options=SHORT)
    with pytest.raises(AcgError) as e:
        bad(B[:, 0] if k == 1 else B, tol=1e-8, precision=precision)
    assert e.value.code == -4, e.value  # ACG_ERR_TIMEOUT
    bad.close()
    good = acgpu.DeviceLapSolver(a, ldli)
    X = good(B, tol=1e-8, precision=precision)
    for c in range(k):
        b = B[:, c] - B[:, c].mean()
        assert good.last_info[c].status == 0
        assert O.relres(a, X[:, c], b) <= 1.01e-8 or precision == "fp64"
    good.close()


def test_the_preconditioner_entry_reports_the_timeout(problem):
    a, ldli = problem
    bad = acgpu.DeviceLapSolver(a, ldli, options=SHORT)
    with pytest.raises(AcgError) as e:
        bad.ldlsolve(np.ones(a.shape[0]))
    assert e.value.code == -4
    bad.close()


@pytest.mark.parametrize("bad_value", [float("nan"), float("inf")])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_non_finite_right_hand_side_is_invalid(problem, bad_value, precision):
    a, ldli = problem
    n = a.shape[0]
    dev = acgpu.DeviceLapSolver(a, ldli)
    b = np.random.default_rng(2).standard_normal(n)
    b[7] = bad_value
    with pytest.raises(AcgError) as e:
        dev(b, tol=1e-8, precision=precision)
    assert e.value.code == -1 and "NaN or infinite" in str(e.value)
    # batched: only the poisoned column is an error; the call reports it
    B = np.random.default_rng(3).standard_normal((n, 8))
    B[3, 5] = bad_value
    with pytest.raises(AcgError):
        dev(B, tol=1e-8, precision=precision)
    # and the solver still works
    x = dev(np.random.default_rng(4).standard_normal(n), tol=1e-8, precision=precision)
    assert np.all(np.isfinite(x))
    dev.close()


def test_non_finite_right_hand_side_in_a_group(gpu_ok):
    graphs = [G.grid2(20, weights="loguniform", seed=s) for s in (1, 2, 3)]
    acgpu.seed(9)
    gs = acgpu.GroupSolver(graphs)
    bs = [np.random.default_rng(s).standard_normal(g.shape[0]) for s, g in enumerate(graphs)]
    bs[1][4] = float("nan")
    with pytest.raises(AcgError) as e:
        gs(bs, tol=1e-8)
    assert e.value.code == -1
    gs.close()
