"""Graph and factor files.

* IJV text, as the reference reads and writes graphs (src/IO.jl:28-83):
  `read_graph` takes one edge per line, "i j" or "i j w", separated by
  whitespace or commas (detected from the first line), 1-based, and returns
  the symmetric adjacency `sparse(i, j, w, n, n) + its transpose` with n the
  largest index; `write_ijv` writes the upper triangle, one "i,j,w" line per
  entry in column-major order (`findnz(triu(mat))`).
* The binary LDLinv file of include/acgpu.h (acg_ldlinv_save / acg_ldlinv_load):
  a factor computed once (here, or by the reference's own elimination on a
  Julia host) is handed over or cached without recomputing it.
"""
from __future__ import annotations

import os

import numpy as np
import scipy.sparse as sp

from ._lib import check, lib
from .solvers import LDLinv, _take_factor

__all__ = ["read_graph", "write_ijv", "writeIJV", "save_ldlinv", "load_ldlinv"]


def read_graph(fn) -> sp.csc_matrix:
    """`read_graph(fn)` (src/IO.jl:28-61): the adjacency matrix of an IJ or IJV
    edge list.  Repeated edges add up, as `sparse` sums duplicates, and an edge
    listed in both directions counts twice, as in the reference."""
    with open(fn) as fh:
        first = fh.readline()
    sep = "," if "," in first else None
    rows = []
    with open(fn) as fh:
        for line in fh:
            line = line.strip()
            if not line:
                continue
            parts = [t for t in (line.split(",") if sep else line.split()) if t.strip() != ""]
            rows.append(parts)
    if not rows:
        raise ValueError(f"{fn}: no edges")
    width = len(rows[0])
    if width not in (2, 3) or any(len(r) != width for r in rows):
        raise ValueError(f"{fn}: every line must hold 2 or 3 fields, the same number throughout")
    ij = np.array([[float(r[0]), float(r[1])] for r in rows])
    if np.any(ij != np.round(ij)) or np.any(ij < 1):
        raise ValueError(f"{fn}: vertex indices must be integers >= 1")
    ij = ij.astype(np.int64)
    w = np.array([float(r[2]) for r in rows]) if width == 3 else np.ones(len(rows))
    n = int(ij.max())
    a = sp.csc_matrix((w, (ij[:, 0] - 1, ij[:, 1] - 1)), shape=(n, n))
    a = (a + a.T).tocsc()
    a.sum_duplicates()
    a.sort_indices()
    return a


def _fmt(v: float) -> str:
    """Shortest decimal string that reads back to the same double, with an
    integral value written as "k.0" (Julia prints Float64 that way)."""
    r = repr(float(v))
    if "e" in r:
        m, e = r.split("e")
        if "." not in m:
            m += ".0"
        return f"{m}e{int(e)}"
    if "." not in r and r not in ("inf", "-inf", "nan"):
        r += ".0"
    return r


def write_ijv(fn, mat) -> None:
    """`writeIJV(filename, mat)` (src/IO.jl:64-83): one "i,j,v" line per
    entry of triu(mat), in column-major order, 1-based.  Values are written
    with enough digits to read back bit for bit."""
    u = sp.triu(sp.csc_matrix(mat), format="csc")
    u.sum_duplicates()
    u.sort_indices()
    u.eliminate_zeros()
    cols = np.repeat(np.arange(u.shape[1]), np.diff(u.indptr))
    with open(fn, "w") as fh:
        for i, j, v in zip(u.indices, cols, u.data):
            fh.write(f"{i + 1},{j + 1},{_fmt(v)}\n")


writeIJV = write_ijv


def save_ldlinv(fn, ldli: LDLinv) -> None:
    """Write `ldli` as a binary LDLinv file (acg_ldlinv_save)."""
    check(lib().acg_ldlinv_save(os.fsencode(fn), ldli.n, np.ascontiguousarray(ldli.col, np.int64),
                                np.ascontiguousarray(ldli.colptr, np.int64),
                                np.ascontiguousarray(ldli.rowval, np.int64),
                                np.ascontiguousarray(ldli.fval, np.float64), np.ascontiguousarray(ldli.d, np.float64),
                                ldli.nnz))


def load_ldlinv(fn) -> LDLinv:
    """Read a binary LDLinv file (acg_ldlinv_load); the library checks its
    header, size and structure."""
    import ctypes
    h = ctypes.c_void_p()
    check(lib().acg_ldlinv_load(os.fsencode(fn), ctypes.byref(h)))
    return _take_factor(h)
