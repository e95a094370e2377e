"""Host elimination (product C++) against the independent Python restatement
of approxChol / ApproxCholPQ / Julia's QuickSort and rand() (oracle), bit for bit."""
import numpy as np
import pytest

import acgpu
from acgpu import generators as G
import approxchol_ref
from julia_rng import JuliaRng


def _ref_factor(a, seed):
    a = acgpu.solvers._csc(a)
    cp = (a.indptr + 1).tolist()
    rv = (a.indices + 1).tolist()
    return approxchol_ref.approx_chol(cp, rv, a.data.tolist(), JuliaRng(seed))


CASES = [
    ("path7", lambda: G.path_graph(7)),
    ("star9", lambda: G.star_graph(9)),
    ("cycle12w", lambda: G.cycle_graph(12, np.linspace(0.5, 2.0, 12))),
    ("complete8", lambda: G.complete_graph(8)),
    ("grid2_9x7", lambda: G.grid2(9, 7)),
    ("grid2_12_logw", lambda: G.grid2(12, weights="loguniform", seed=3)),
    ("grid3_5", lambda: G.grid3(5)),
    ("tree60", lambda: G.random_tree(60, seed=5)),
    ("pm_200", lambda: G.path_plus_matchings(200, k=4, sigma=2.0, seed=1)),
    ("rgg_300", lambda: _largest_comp(G.random_geometric(300, seed=2))),
]


def _largest_comp(a):
    co = acgpu.components(a)
    big = np.argmax(np.bincount(co))
    ind = np.where(co == big)[0]
    return a[ind][:, ind]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("seed", [1, 7])
def test_factor_matches_restatement(name, make, seed):
    a = make()
    acgpu.seed(seed)
    f = acgpu.approx_chol(a)
    col, colptr, rowval, fval, d = _ref_factor(a, seed)
    np.testing.assert_array_equal(f.col, col)
    np.testing.assert_array_equal(f.colptr, colptr)
    np.testing.assert_array_equal(f.rowval, rowval)
    assert np.array_equal(f.fval, fval), "fval differs bitwise"
    assert np.array_equal(f.d, d), "d differs bitwise"


def test_factor_shape_invariants():
    a = G.grid2(30, weights="loguniform", seed=4)
    acgpu.seed(3)
    f = acgpu.approx_chol(a)
    n = a.shape[0]
    assert sorted(set(f.col.tolist())) == sorted(set(range(1, n + 1)) - {int(np.setdiff1d(np.arange(1, n + 1), f.col)[0])})
    assert f.colptr[0] == 1 and f.colptr[-1] == f.nnz + 1
    assert np.all(np.diff(f.colptr) >= 1)
    assert np.all((f.fval > 0) & (f.fval <= 1))
    # the last entry of every column has fval == 1 (src/approxChol.jl:964-966)
    assert np.all(f.fval[f.colptr[1:] - 2] == 1.0)
    root = np.setdiff1d(np.arange(1, n + 1), f.col)[0]
    assert f.d[root - 1] == 0.0 and np.all(np.delete(f.d, root - 1) > 0)


def test_seed_stream_advances_like_global_rng():
    a = G.grid2(10)
    acgpu.seed(11)
    f1 = acgpu.approx_chol(a)
    f2 = acgpu.approx_chol(a)  # continues the stream: a different factor
    acgpu.seed(11)
    f3 = acgpu.approx_chol(a)
    assert np.array_equal(f1.fval, f3.fval)
    assert not np.array_equal(f1.fval, f2.fval)


def test_negative_weight_rejected():
    a = G.grid2(4).tolil()
    a[0, 1] = a[1, 0] = -1.0
    with pytest.raises(Exception):
        acgpu.approx_chol(a.tocsc())


def _ref_ordered(a, order, seed):
    """The restatement's factor for a fixed order: the permutation comes from
    the product's stream (as approx_chol draws it), the elimination from the
    restatement continuing that stream."""
    from acgpu.solvers import elimination_order
    a = acgpu.solvers._csc(a)
    acgpu.seed(seed)
    p = elimination_order(a, order)
    rng = JuliaRng(state=[int(x) for x in acgpu.rng_state()])
    cp = (a.indptr + 1).tolist()
    rv = (a.indices + 1).tolist()
    return approxchol_ref.approx_chol_ord(cp, rv, a.data.tolist(), rng, None if p is None else p.tolist())


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("order", ["given", "wdeg", "random"])
def test_ordered_factor_matches_restatement(name, make, order):
    a = make()
    ref = _ref_ordered(a, order, 11)
    acgpu.seed(11)
    f = acgpu.approx_chol(a, acgpu.ApproxCholParams(order=order))
    got = (f.col, f.colptr, f.rowval, f.fval, f.d)
    for x, y, what in zip(got, ref, ("col", "colptr", "rowval", "fval", "d")):
        assert np.array_equal(np.asarray(x), np.asarray(y)), what
    n = a.shape[0]
    # a valid elimination order: every vertex but one eliminated once, F = colptr[end] - 1
    assert len(set(f.col.tolist())) == n - 1 and f.colptr[-1] - 1 == f.fval.shape[0]


def test_given_order_eliminates_in_index_order():
    a = G.grid2(6, 5)
    acgpu.seed(2)
    f = acgpu.approx_chol(a, acgpu.ApproxCholParams(order="given"))
    assert f.col.tolist() == list(range(1, a.shape[0]))


def test_other_orders_are_the_given_order():
    # the reference's dispatch sends any order but :deg/:wdeg/:random to
    # approxchol_lapGiven (src/approxChol.jl:1836-1850)
    a = G.grid2(5)
    acgpu.seed(3)
    f1 = acgpu.approx_chol(a, acgpu.ApproxCholParams(order="bogus"))
    acgpu.seed(3)
    f2 = acgpu.approx_chol(a, acgpu.ApproxCholParams(order="given"))
    assert np.array_equal(f1.fval, f2.fval) and np.array_equal(f1.rowval, f2.rowval)


def _ref_split(a, seed, split, merge):
    a = acgpu.solvers._csc(a)
    cp = (a.indptr + 1).tolist()
    rv = (a.indices + 1).tolist()
    return approxchol_ref.approx_chol_split(cp, rv, a.data.tolist(), JuliaRng(seed), split, merge)


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("split,merge", [(2, 2), (3, 2), (2, 1), (2, 0), (3, 0)])
def test_split_merge_factor_matches_restatement(name, make, split, merge):
    a = make()
    ref = _ref_split(a, 5, split, merge)
    acgpu.seed(5)
    f = acgpu.approx_chol(a, acgpu.ApproxCholParams("deg", 5, split, merge))
    got = (f.col, f.colptr, f.rowval, f.fval, f.d)
    for x, y, what in zip(got, ref, ("col", "colptr", "rowval", "fval", "d")):
        assert np.array_equal(np.asarray(x), np.asarray(y)), what
    n = a.shape[0]
    assert len(set(f.col.tolist())) == n - 1 and f.colptr[-1] - 1 == f.fval.shape[0]


@pytest.mark.parametrize("split", [2, 3])
def test_split_without_merge_is_an_unreached_cap(split):
    """approxChol(llmat, split) (merge < 1) averages parallel edges like
    compressAvgCol! with a cap no vertex reaches: the factor equals the merge
    form with merge >= the largest multiplicity, and differs from a low cap."""
    a = G.grid2(12, weights="loguniform", seed=3)
    fs = []
    for merge in (0, 10 ** 9, 1):
        acgpu.seed(9)
        fs.append(acgpu.approx_chol(a, acgpu.ApproxCholParams("deg", 5, split, merge)))
    assert np.array_equal(fs[0].fval, fs[1].fval) and np.array_equal(fs[0].rowval, fs[1].rowval)
    assert not (fs[0].fval.shape == fs[2].fval.shape and np.array_equal(fs[0].fval, fs[2].fval))
