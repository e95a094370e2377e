"""The autotuner's search (coordinate descent over acg_options knobs) on
synthetic cost functions (no device), and on the device against a real graph."""
import numpy as np
import pytest

import acgpu
from acgpu import generators as G
from acgpu.tuning import coordinate_descent, default_space, autotune
import oracle as O


def test_descent_finds_separable_minimum():
    space = {"a": [0, 1, 2, 3], "b": [0, 10, 20]}
    cost = lambda o: 5.0 + (o["a"] - 2) ** 2 + 0.01 * (o["b"] - 20) ** 2
    res = coordinate_descent(cost, space)
    assert res.options == {"a": 2, "b": 20}
    assert res.ms == pytest.approx(5.0)
    assert res.baseline_ms == pytest.approx(cost({"a": 0, "b": 0}))
    assert res.speedup > 1.0


def test_descent_keeps_defaults_within_min_gain():
    space = {"a": [0, 1, 2]}
    res = coordinate_descent(lambda o: 10.0 - 0.1 * o["a"], space, min_gain=0.05)
    assert res.options == {}  # 2 % faster is below the 5 % bar
    res = coordinate_descent(lambda o: 10.0 - 1.0 * o["a"], space, min_gain=0.05)
    assert res.options == {"a": 2}


def test_descent_measures_each_candidate_once():
    calls = []
    space = {"a": [0, 1], "b": [0, 1]}

    def cost(o):
        calls.append(dict(o))
        return 1.0 + o["a"] + o["b"]

    res = coordinate_descent(cost, space, rounds=3)
    keys = [tuple(sorted(c.items())) for c in calls]
    assert len(keys) == len(set(keys))
    assert res.options == {} and len(res.trials) == len(calls)


def test_default_spaces_start_at_defaults():
    for k in (1, 64):
        sp = default_space(k)
        assert all(v[0] == 0 for v in sp.values())
        known = {f[0] for f in acgpu._lib.AcgOptions._fields_}
        assert set(sp) <= known


@pytest.mark.gpu
def test_autotune_on_device(gpu_ok):
    a = G.grid3(18, weights="loguniform", seed=41)
    acgpu.seed(1)
    ldli = acgpu.approx_chol(a)
    space = {"dense_tail": [0, 512, -1], "batch_bwd_heavy": [0, 16]}
    res = autotune(a, ldli, nrhs=16, precision="mixed", space=space, reps=2)
    assert res.ms > 0 and res.ms <= res.baseline_ms * 1.0000001
    assert len(res.trials) >= 3
    dev = acgpu.DeviceLapSolver(a, ldli, options=res.options)
    B = np.random.default_rng(2).standard_normal((a.shape[0], 16))
    X = dev(B, tol=1e-8, maxits=2000, precision="mixed")
    for c in range(16):
        assert O.relres(a, X[:, c], B[:, c] - B[:, c].mean()) <= 1e-8 * 1.01
    dev.close()
