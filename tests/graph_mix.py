"""Seeded "mixed recipe" graphs for the reference's randomized solver tests.

The reference tests its solvers on `wted_chimera(n, k)` graphs
(test/testSolvers.jl:103-107,155-205): a connected graph on exactly n
vertices built from a random recipe of smaller generators (joins of two
graphs by a few random edges, grids, products, random regular-like and
geometric graphs, trees) with one of several random weightings (unit,
uniform, wide log-scale spreads, weights from differences of smoothed random
potentials).  That generator draws from Julia's `rand`/`randn`/`randperm`
streams and cannot be reproduced without Julia, so these tests use this
module's own recipe graphs of the same kind and size instead.  They are
connected, have exactly n vertices and are deterministic for a seed.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components

from acgpu import generators as G


def _edges(a):
    c = sp.triu(sp.coo_matrix(a), k=1)
    return c.row.astype(np.int64), c.col.astype(np.int64)


def _connect(n, i, j, rng):
    """Add one edge between consecutive components (in a random order) so the
    graph is connected."""
    if n < 2:
        return i, j
    a = sp.coo_matrix((np.ones(i.shape[0]), (i, j)), shape=(n, n))
    nc, lab = connected_components(a, directed=False)
    if nc == 1:
        return i, j
    reps = np.array([rng.choice(np.where(lab == c)[0]) for c in rng.permutation(nc)], dtype=np.int64)
    return np.concatenate([i, reps[:-1]]), np.concatenate([j, reps[1:]])


def _base(n, rng):
    kind = rng.integers(6)
    if n <= 3 or kind == 0:  # random tree
        parent = np.array([rng.integers(0, v) for v in range(1, n)], dtype=np.int64)
        return np.arange(1, n, dtype=np.int64), parent
    if kind == 1:  # path over a permutation plus matchings
        p = rng.permutation(n)
        ii, jj = [p[:-1]], [p[1:]]
        for _ in range(int(rng.integers(1, 4))):
            q = rng.permutation(n)
            h = n // 2
            ii.append(q[:h])
            jj.append(q[h:2 * h])
        return np.concatenate(ii), np.concatenate(jj)
    if kind == 2:  # sparse Erdos-Renyi
        deg = rng.uniform(2.0, 8.0)
        m = int(deg * n / 2)
        return rng.integers(0, n, m), rng.integers(0, n, m)
    if kind == 3:  # random geometric
        a = G.random_geometric(n, mean_degree=float(rng.uniform(4, 10)), seed=int(rng.integers(1 << 30)),
                               weights="lognormal:1")
        return _edges(a)
    if kind == 4:  # cycle with chords
        i = np.arange(n, dtype=np.int64)
        k = int(rng.integers(0, max(1, n // 4)))
        return np.concatenate([i, rng.integers(0, n, k)]), np.concatenate([(i + 1) % n, rng.integers(0, n, k)])
    # dense-ish small block
    if n <= 60:
        iu, ju = np.triu_indices(n, 1)
        keep = rng.random(iu.shape[0]) < rng.uniform(0.2, 1.0)
        return iu[keep].astype(np.int64), ju[keep].astype(np.int64)
    return _base(n, rng)


def _recipe(n, rng, depth=0):
    """Undirected edge list (i, j) of a random recipe graph on n vertices."""
    if n < 30 or depth > 3 or rng.random() < 0.2:
        return _base(n, rng)
    r = rng.random()
    if r < 0.35 or n < 200:
        # two smaller recipe graphs joined by k random edges
        n1 = 10 + int((n - 20) * rng.random())
        n2 = n - n1
        k = int(np.ceil(np.exp(rng.random() * np.log(max(2.0, min(n1, n2) / 2)))))
        i1, j1 = _recipe(n1, rng, depth + 1)
        i2, j2 = _recipe(n2, rng, depth + 1)
        ci, cj = rng.integers(0, n1, k), n1 + rng.integers(0, n2, k)
        return np.concatenate([i1, i2 + n1, ci]), np.concatenate([j1, j2 + n1, cj])
    if r < 0.6:
        # a 2D or 3D grid on the largest box that fits, the rest hung on as a recipe graph
        if rng.random() < 0.5:
            s = int(np.floor(np.sqrt(n)))
            a = G.grid2(s, max(1, n // s))
        else:
            s = int(np.floor(n ** (1 / 3)))
            a = G.grid3(s, s, max(1, n // (s * s)))
        ng = a.shape[0]
        i, j = _edges(a)
        if ng < n:
            ir, jr = _recipe(n - ng, rng, depth + 1) if n - ng >= 2 else (np.zeros(0, np.int64), np.zeros(0, np.int64))
            k = int(rng.integers(1, 4))
            i = np.concatenate([i, ir + ng, rng.integers(0, ng, k)])
            j = np.concatenate([j, jr + ng, ng + rng.integers(0, n - ng, k)])
        return i, j
    if r < 0.8:
        # product of two smaller recipe graphs, the remainder joined on
        n1 = int(rng.integers(2, max(3, int(np.sqrt(n)))))
        n2 = n // n1
        i1, j1 = _recipe(n1, rng, depth + 1)
        i2, j2 = _recipe(n2, rng, depth + 1)
        a1 = sp.coo_matrix((np.ones(i1.shape[0]), (i1, j1)), shape=(n1, n1))
        a2 = sp.coo_matrix((np.ones(i2.shape[0]), (i2, j2)), shape=(n2, n2))
        a1 = ((a1 + a1.T) > 0).astype(float)
        a2 = ((a2 + a2.T) > 0).astype(float)
        prod = sp.kron(a1, sp.identity(n2)) + sp.kron(sp.identity(n1), a2)
        i, j = _edges(prod)
        ng = n1 * n2
        if ng < n:
            k = int(rng.integers(1, 4))
            extra = np.arange(ng, n, dtype=np.int64)
            i = np.concatenate([i, extra, rng.integers(0, ng, k)])
            j = np.concatenate([j, rng.integers(0, ng, extra.shape[0]), ng + rng.integers(0, n - ng, k)])
        return i, j
    return _base(n, rng)


def _weights(n, i, j, rng):
    m = i.shape[0]
    r = rng.random()
    if r < 0.2:
        return np.ones(m)
    if r < 0.4:
        return rng.random(m) + 1e-12
    if r < 0.6:
        # log-scale spread of up to 8 decades
        return np.exp(rng.uniform(-np.log(10.0) * rng.uniform(1, 8), 0.0, m))
    if r < 0.75:
        return rng.lognormal(0.0, rng.uniform(0.5, 3.0), m)
    # differences of a random potential, optionally smoothed by random-walk steps
    a = sp.coo_matrix((np.ones(m), (i, j)), shape=(n, n))
    a = (a + a.T).tocsr()
    deg = np.maximum(np.asarray(a.sum(axis=1)).ravel(), 1.0)
    v = rng.standard_normal(n)
    for _ in range(int(rng.integers(0, 10))):
        v = a @ (v / deg)
        v -= v.mean()
    w = np.abs(v[i] - v[j])
    w = w ** rng.uniform(0.5, 2.0)
    return np.maximum(w, 1e-8 * max(w.max(), 1e-300)) + 1e-300


def mixed_graph(n: int, seed: int, weighted: bool = True) -> sp.csc_matrix:
    """A connected recipe graph on exactly n vertices (see the module doc)."""
    rng = np.random.default_rng(seed)
    i, j = _recipe(n, rng)
    keep = i != j
    i, j = i[keep], j[keep]
    i, j = _connect(n, i, j, rng)
    p = rng.permutation(n)
    i, j = p[i], p[j]
    # one record per undirected edge, so both triangles get the same weight
    lo, hi = np.minimum(i, j), np.maximum(i, j)
    key = np.unique(lo * n + hi)
    i, j = key // n, key % n
    w = _weights(n, i, j, rng) if weighted else None
    return G.from_edges(n, i, j, w)


def disjoint_union(graphs) -> sp.csc_matrix:
    """`disjoin(a, b)` of the reference: the block-diagonal union."""
    a = sp.block_diag(graphs, format="csc")
    a.sort_indices()
    return a
