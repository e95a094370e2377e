"""Seeded graph generators for the solve-phase workloads.

Every generator returns a symmetric ``scipy.sparse.csc_matrix`` adjacency
matrix (zero diagonal, sorted row indices, float64 weights), the same object
the reference passes to ``approxchol_lap``.

Vertex numbering follows the reference's grid builders: ``grid2(n, m)`` is
``product_graph(path_graph(n), path_graph(m))`` and ``grid3(n1, n2, n3)`` is
``product_graph(path_graph(n1), product_graph(path_graph(n2), path_graph(n3)))``
(src/graphGenerators.jl:219-241, src/graphOps.jl:157-184), so the last
coordinate varies fastest.  Weighted variants draw one weight per edge from a
numpy ``Generator`` seeded explicitly.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

__all__ = [
    "from_edges", "path_graph", "grid2", "grid3", "rand_matching_edges",
    "path_plus_matchings", "random_geometric", "cycle_graph", "star_graph",
    "complete_graph", "random_tree", "loguniform_weights", "lognormal_weights", "largest_component",
]


def from_edges(n: int, i, j, w=None) -> sp.csc_matrix:
    """Symmetric adjacency from an undirected edge list; duplicates are summed
    like ``sparse(i, j, v, n, n)`` (src/IJV.jl:67)."""
    i = np.asarray(i, dtype=np.int64)
    j = np.asarray(j, dtype=np.int64)
    if w is None:
        w = np.ones(i.shape[0], dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    keep = i != j
    i, j, w = i[keep], j[keep], w[keep]
    a = sp.coo_matrix((np.concatenate([w, w]), (np.concatenate([i, j]), np.concatenate([j, i]))),
                      shape=(n, n)).tocsc()
    a.sum_duplicates()
    a.sort_indices()
    return a


def _grid_edges(dims):
    dims = list(dims)
    n = int(np.prod(dims))
    idx = np.arange(n, dtype=np.int64).reshape(dims)
    ii, jj = [], []
    for ax in range(len(dims)):
        lo = [slice(None)] * len(dims)
        hi = [slice(None)] * len(dims)
        lo[ax] = slice(0, dims[ax] - 1)
        hi[ax] = slice(1, dims[ax])
        ii.append(idx[tuple(lo)].ravel())
        jj.append(idx[tuple(hi)].ravel())
    return n, np.concatenate(ii), np.concatenate(jj)


def lognormal_weights(m: int, sigma: float, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).lognormal(0.0, sigma, size=m)


def _weights(kind: str, m: int, seed: int):
    if kind == "unit":
        return None
    if kind == "loguniform":
        return loguniform_weights(m, 1e-3, 1.0, seed)
    if kind.startswith("lognormal"):
        sigma = float(kind.split(":")[1]) if ":" in kind else 1.0
        return lognormal_weights(m, sigma, seed)
    raise ValueError(f"unknown weights {kind!r}")


def loguniform_weights(m: int, lo: float, hi: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=m))


def path_graph(n: int) -> sp.csc_matrix:
    i = np.arange(n - 1)
    return from_edges(n, i, i + 1)


def cycle_graph(n: int, weights=None) -> sp.csc_matrix:
    i = np.arange(n)
    return from_edges(n, i, (i + 1) % n, weights)


def star_graph(n: int) -> sp.csc_matrix:
    return from_edges(n, np.zeros(n - 1, dtype=np.int64), np.arange(1, n))


def complete_graph(n: int) -> sp.csc_matrix:
    i, j = np.triu_indices(n, 1)
    return from_edges(n, i, j)


def random_tree(n: int, seed: int, weighted: bool = True) -> sp.csc_matrix:
    rng = np.random.default_rng(seed)
    parent = np.array([rng.integers(0, v) for v in range(1, n)], dtype=np.int64)
    w = rng.lognormal(0.0, 1.0, n - 1) if weighted else None
    return from_edges(n, np.arange(1, n), parent, w)


def grid2(n: int, m: int | None = None, weights: str = "unit", seed: int = 0) -> sp.csc_matrix:
    """n-by-m grid (4-neighbour). ``weights``: "unit", "loguniform" in [1e-3, 1],
    or "lognormal[:sigma]"."""
    m = n if m is None else m
    nv, i, j = _grid_edges((n, m))
    return from_edges(nv, i, j, _weights(weights, i.shape[0], seed))


def grid3(n1: int, n2: int | None = None, n3: int | None = None, weights: str = "unit",
          seed: int = 0) -> sp.csc_matrix:
    """n1-by-n2-by-n3 grid (6-neighbour). ``weights``: "unit", "loguniform" in
    [1e-3, 1], or "lognormal[:sigma]"."""
    n2 = n1 if n2 is None else n2
    n3 = n1 if n3 is None else n3
    nv, i, j = _grid_edges((n1, n2, n3))
    return from_edges(nv, i, j, _weights(weights, i.shape[0], seed))


def rand_matching_edges(n: int, rng: np.random.Generator):
    p = rng.permutation(n)
    h = n // 2
    return p[:h], p[h:2 * h]


def path_plus_matchings(n: int, k: int = 4, sigma: float = 2.0, seed: int = 0) -> sp.csc_matrix:
    """A path over a random vertex permutation plus ``k`` random perfect
    matchings; lognormal(0, sigma) weights; parallel edges merge by summation."""
    rng = np.random.default_rng(seed)
    p = rng.permutation(n)
    ii = [p[:-1]]
    jj = [p[1:]]
    for _ in range(k):
        a, b = rand_matching_edges(n, rng)
        ii.append(a)
        jj.append(b)
    i = np.concatenate(ii)
    j = np.concatenate(jj)
    w = rng.lognormal(0.0, sigma, i.shape[0])
    return from_edges(n, i, j, w)


def largest_component(a) -> sp.csc_matrix:
    from scipy.sparse.csgraph import connected_components
    _, lab = connected_components(a, directed=False)
    big = np.argmax(np.bincount(lab))
    ind = np.where(lab == big)[0]
    sub = sp.csc_matrix(a[ind][:, ind])
    sub.sort_indices()
    return sub


def random_geometric(n: int, mean_degree: float = 8.0, seed: int = 0, weights: str = "inverse_distance") -> sp.csc_matrix:
    """Points uniform in the unit square joined within radius sqrt(d/(pi n));
    weights 1/distance (or "lognormal[:sigma]").  May be disconnected."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    r = np.sqrt(mean_degree / (np.pi * n))
    pairs = cKDTree(pts).query_pairs(r, output_type="ndarray")
    i, j = pairs[:, 0].astype(np.int64), pairs[:, 1].astype(np.int64)
    if weights == "inverse_distance":
        dist = np.linalg.norm(pts[i] - pts[j], axis=1)
        w = 1.0 / np.maximum(dist, 1e-12)
    else:
        w = _weights(weights, i.shape[0], seed + 1)
    return from_edges(n, i, j, w)
