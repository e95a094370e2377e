"""Failure handling that needs no GPU: acg_create rejects malformed inputs with
ACG_ERR_INVALID before it touches a device.

The reference raises Julia exceptions for bad inputs (src/approxChol.jl:1533,
"Adjacency matrix can not have negative edge weights"); the C ABI returns
ACG_ERR_INVALID with a message instead.  Every case here is checked on the
host, so the tests run (and give the same answer) without a GPU.  The GPU
side of failure handling, a bounded sweep wait that runs out, is in
test_gpu_failure.py.
"""
import ctypes

import numpy as np
import pytest

import acgpu
from acgpu import generators as G
from acgpu._lib import lib

ERR_INVALID = -1


def _problem():
    a = G.grid2(6, weights="loguniform", seed=2)
    acgpu.seed(4)
    f = acgpu.approx_chol(a)
    return a, f


def _create(a, col, colptr, rowval, fval, d, nzval=None):
    h = ctypes.c_void_p()
    L = lib()
    rc = L.acg_create(a.shape[0], a.indptr.astype(np.int64), a.indices.astype(np.int64),
                      np.ascontiguousarray(a.data if nzval is None else nzval), np.ascontiguousarray(col),
                      np.ascontiguousarray(colptr), np.ascontiguousarray(rowval), np.ascontiguousarray(fval),
                      np.ascontiguousarray(d), fval.shape[0], 1, None, ctypes.byref(h))
    if rc == 0:
        L.acg_destroy(h)
    return rc, L.acg_last_error().decode()


def test_a_valid_factor_passes_the_host_checks():
    import torch
    a, f = _problem()
    rc, msg = _create(a, f.col, f.colptr, f.rowval, f.fval, f.d)
    # without a device the checks pass and only the device check fails
    assert rc == (0 if torch.cuda.is_available() else -5), msg


def test_non_permutation_col_is_rejected():
    a, f = _problem()
    col = f.col.copy()
    col[3] = col[2]
    rc, msg = _create(a, col, f.colptr, f.rowval, f.fval, f.d)
    assert rc == ERR_INVALID and "repeats a vertex" in msg


@pytest.mark.parametrize("bad", [1.5, -0.25, float("nan")])
def test_fval_outside_unit_interval_is_rejected(bad):
    a, f = _problem()
    fval = f.fval.copy()
    fval[5] = bad
    rc, msg = _create(a, f.col, f.colptr, f.rowval, fval, f.d)
    assert rc == ERR_INVALID and "fval" in msg


def test_rowval_against_the_elimination_order_is_rejected():
    a, f = _problem()
    rowval = f.rowval.copy()
    rowval[-1] = f.col[0]  # the first eliminated vertex cannot appear in the last column
    rc, msg = _create(a, f.col, f.colptr, rowval, f.fval, f.d)
    assert rc == ERR_INVALID and "elimination order" in msg


@pytest.mark.parametrize("bad", [-1.0, float("inf"), float("nan")])
def test_bad_diagonal_is_rejected(bad):
    a, f = _problem()
    d = f.d.copy()
    d[0] = bad
    rc, msg = _create(a, f.col, f.colptr, f.rowval, f.fval, d)
    assert rc == ERR_INVALID and "ldli.d" in msg


def test_empty_column_is_rejected():
    a, f = _problem()
    colptr = f.colptr.copy()
    colptr[2] = colptr[1]
    rc, msg = _create(a, f.col, colptr, f.rowval, f.fval, f.d)
    assert rc == ERR_INVALID


@pytest.mark.parametrize("bad", [-2.0, float("inf")])
def test_bad_edge_weight_is_rejected(bad):
    a, f = _problem()
    nz = a.data.copy()
    nz[0] = bad
    rc, msg = _create(a, f.col, f.colptr, f.rowval, f.fval, f.d, nzval=nz)
    assert rc == ERR_INVALID and "negative edge weights" in msg


def test_group_with_a_column_across_graphs_is_rejected():
    import scipy.sparse as sp
    gs = [G.grid2(5, weights="loguniform", seed=s) for s in (1, 2)]
    acgpu.seed(7)
    fs = [acgpu.approx_chol(g) for g in gs]
    u = sp.block_diag(gs, format="csc")
    u.sort_indices()
    off = np.array([0, 25, 50], np.int64)
    col = np.concatenate([fs[0].col, fs[1].col + 25]).astype(np.int64)
    colptr = np.concatenate([fs[0].colptr[:-1], fs[1].colptr[:-1] + fs[0].nnz, [fs[0].nnz + fs[1].nnz + 1]])
    rowval = np.concatenate([fs[0].rowval, fs[1].rowval + 25]).astype(np.int64)
    rowval[0] = 26 + fs[1].col[-1] - 1  # graph 0's first column names a late vertex of graph 1
    fval = np.concatenate([fs[0].fval, fs[1].fval])
    d = np.concatenate([fs[0].d, fs[1].d])
    h = ctypes.c_void_p()
    rc = lib().acg_create_group(2, off, 50, u.indptr.astype(np.int64), u.indices.astype(np.int64),
                                np.ascontiguousarray(u.data), col, col.shape[0], colptr.astype(np.int64), rowval,
                                fval, d, fval.shape[0], 1, None, ctypes.byref(h))
    assert rc == ERR_INVALID and b"two different graphs" in lib().acg_last_error()
