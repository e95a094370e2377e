"""Host-side mirror of Laplacians.jl's `approxchol_lap` solver interface.

    f = approxchol_lap(a; tol=1e-6, maxits=1000, maxtime=Inf, verbose=false,
                       pcgIts=Int[], params=ApproxCholParams())
    x = f(b; tol, maxits, maxtime, verbose, pcgIts)

(src/approxChol.jl:1522-1545, 1581-1626; kwarg semantics in
docs/src/usingSolvers.md:102-113.)  Here ``a`` is a symmetric
``scipy.sparse`` adjacency matrix and ``f`` is a callable whose solves run on
the GPU through libacgpu.so.  Every keyword keeps its meaning: ``pcgIts`` is a
list whose first entry receives the iteration count, keywords given to ``f``
override the ones given at construction, and a disconnected graph is solved
per component as `lapWrapComponents` does (src/solverInterface.jl:212-275).

Extra keyword (not in the reference): ``precision`` = "fp64" (default; the
reference algorithm in FP64 on the GPU) or "mixed" (FP32 PCG inside FP64
iterative refinement on the true residual).
"""
from __future__ import annotations

import ctypes
import math
import os
import time
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import AcgOptions, AcgSolveInfo, AcgStats, check, lib

__all__ = [
    "ApproxCholParams", "LDLinv", "approxchol_lap", "approxchol_lap1", "lap", "seed", "rng_state",
    "set_rng_state", "approx_chol", "components", "vec_to_comps", "DeviceLapSolver", "GroupSolver", "null_solver",
    "ServeLoop", "Ticket", "approx_chol_parallel",
]

_PRECISIONS = {"fp64": 0, "mixed": 1}

# ---- the global random stream (Julia's default RNG) -------------------------

_RNG = np.zeros(4, dtype=np.uint64)


def seed(s: int) -> None:
    """`Random.seed!(s)`: reseed the stream the elimination draws from."""
    check(lib().acg_rng_seed(int(s), _RNG))


def rng_state() -> np.ndarray:
    return _RNG.copy()


def set_rng_state(state) -> None:
    _RNG[:] = np.asarray(state, dtype=np.uint64)


def _seed_from_entropy():
    # Julia seeds its default generator from system entropy at start-up.
    seed(int.from_bytes(os.urandom(8), "little"))


# ---- parameters and factor ----------------------------------------------------

@dataclass
class ApproxCholParams:
    """`ApproxCholParams(order, stag_test, split, merge)`, default (:deg, 5, 0, 0)
    (src/approxChol.jl:80-90)."""
    order: str = "deg"
    stag_test: int = 5
    split: int = 0
    merge: int = 0


@dataclass
class LDLinv:
    """The factor in the reference layout (src/approxCholTypes.jl:73-79), 1-based."""
    col: np.ndarray
    colptr: np.ndarray
    rowval: np.ndarray
    fval: np.ndarray
    d: np.ndarray

    @property
    def n(self) -> int:
        return int(self.d.shape[0])

    @property
    def nnz(self) -> int:
        return int(self.fval.shape[0])


def _csc(a) -> sp.csc_matrix:
    a = sp.csc_matrix(a, dtype=np.float64)
    a.sum_duplicates()
    a.sort_indices()
    return a


def lap(a) -> sp.csc_matrix:
    """`lap(a) = sparse(Diagonal(a*ones(n))) - a` (src/graphOps.jl:25)."""
    a = _csc(a)
    return _csc(sp.diags(np.asarray(a.sum(axis=1)).ravel()) - a)


def rand(k: int) -> np.ndarray:
    """k draws of Julia's scalar `rand()` from the global stream (one at a time,
    in order; Julia's bulk `rand(k)` fills arrays by another method)."""
    out = np.empty(int(k), dtype=np.float64)
    if k > 0:
        check(lib().acg_rng_rand(_RNG, out, int(k)))
    return out


def elimination_order(a, order: str):
    """The vertex order (1-based; None = the given order 1..n) that the
    reference's fixed-order solvers eliminate in:
      "given"  approxchol_lapGiven   (src/approxChol.jl:1628-1677): 1..n;
      "wdeg"   approxchol_lapWdeg    (src/approxChol.jl:1679-1734): sortperm of
               the weighted degrees times 1 + rand();
      "random" approxchol_lapRandom  (src/approxChol.jl:1736-1789): a uniform
               random permutation (Fisher-Yates on rand(); Julia's randperm
               samples its integers differently)."""
    a = _csc(a)
    n = a.shape[0]
    if order == "wdeg":
        v = np.asarray(a.sum(axis=0), dtype=np.float64).ravel()
        v = v * (1.0 + rand(n))
        return (np.argsort(v, kind="stable") + 1).astype(np.int64)
    if order == "random":
        p = np.arange(1, n + 1, dtype=np.int64)
        u = rand(n - 1)
        for t, i in enumerate(range(n - 1, 0, -1)):
            j = min(int(u[t] * (i + 1)), i)
            p[i], p[j] = p[j], p[i]
        return p
    return None  # any other order is the given one (src/approxChol.jl:1836-1850)


def approx_chol(a, params: ApproxCholParams | None = None) -> LDLinv:
    """The reference's host elimination, drawing from the global stream:
    `approxChol(LLmatp(a))` for the default :deg order (src/approxChol.jl:864-977),
    `approxChol(LLmatp(a, split), split, merge)` for :deg with split, merge >= 1
    (src/approxChol.jl:979-1157; approxchol_lap2 uses 2, 2), `approxChol(LLmatp(a,
    split), split)` for split >= 1, merge < 1 (src/approxChol.jl:1162-1322), and
    `approxChol(LLMatOrd(a[, p]))` for :wdeg, :random and any other order, which
    the reference treats as :given (src/approxChol.jl:758-862, 1791-1851)."""
    a = _csc(a)
    n = a.shape[0]
    params = params or ApproxCholParams()
    order = params.order
    L = lib()
    h = ctypes.c_void_p()
    cp = a.indptr.astype(np.int64) + 1
    rv = a.indices.astype(np.int64) + 1
    if order == "deg" and params.split >= 1:
        # merge < 1: approxChol(llmat, split) (src/approxChol.jl:1162-1322)
        check(L.acg_approxchol_split(n, cp, rv, np.ascontiguousarray(a.data), int(params.split), int(params.merge),
                                     _RNG, ctypes.byref(h)))
    elif order == "deg":
        check(L.acg_approxchol(n, cp, rv, np.ascontiguousarray(a.data), _RNG, ctypes.byref(h)))
    else:
        p = elimination_order(a, order)
        pp = None if p is None else p.ctypes.data_as(ctypes.c_void_p)
        check(L.acg_approxchol_ordered(n, cp, rv, np.ascontiguousarray(a.data), pp, _RNG, ctypes.byref(h)))
    return _take_factor(h)


def approx_chol_parallel(a, seed: int = 1, threads: int | None = None) -> tuple[LDLinv, int]:
    """Opt-in parallel elimination (acg_approxchol_parallel; not in the
    reference): rounds of independent low-degree vertices eliminated at once on
    `threads` host threads (default: all), each with the reference's
    per-vertex step but its own keyed random numbers, so the factor is a
    different sample than approx_chol's.  Returns (factor, rounds); the
    factor's DAG is at most `rounds` levels deep."""
    a = _csc(a)
    n = a.shape[0]
    if threads is None:
        threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    h = ctypes.c_void_p()
    rounds = ctypes.c_int64()
    check(lib().acg_approxchol_parallel(n, a.indptr.astype(np.int64) + 1, a.indices.astype(np.int64) + 1,
                                        np.ascontiguousarray(a.data), int(seed) & ((1 << 64) - 1), int(threads),
                                        ctypes.byref(rounds), ctypes.byref(h)))
    return _take_factor(h), int(rounds.value)


def _take_factor(h) -> LDLinv:
    """Copy a library factor handle (acg_factor) into an LDLinv and free it."""
    L = lib()
    try:
        nn = ctypes.c_int64()
        F = ctypes.c_int64()
        check(L.acg_factor_dims(h, ctypes.byref(nn), ctypes.byref(F)))
        n = nn.value
        col = np.empty(n - 1, np.int64)
        colptr = np.empty(n, np.int64)
        rowval = np.empty(F.value, np.int64)
        fval = np.empty(F.value, np.float64)
        d = np.empty(n, np.float64)
        check(L.acg_factor_export(h, col, colptr, rowval, fval, d))
    finally:
        L.acg_factor_free(h)
    return LDLinv(col, colptr, rowval, fval, d)


# ---- components (src/graphAlgs.jl:64-108, 135-155) ---------------------------

def components(a) -> np.ndarray:
    """Component label (1-based) of every vertex, numbered in order of each
    component's smallest vertex, as `components` does."""
    from scipy.sparse.csgraph import connected_components
    a = _csc(a)
    _, lab = connected_components(a, directed=False)
    first = np.full(lab.max() + 1, a.shape[0], dtype=np.int64)
    np.minimum.at(first, lab, np.arange(a.shape[0]))
    order = np.argsort(first, kind="stable")
    relabel = np.empty_like(order)
    relabel[order] = np.arange(order.shape[0])
    return relabel[lab] + 1


def vec_to_comps(co: np.ndarray) -> list:
    order = np.argsort(co, kind="stable")
    bounds = np.cumsum(np.bincount(co)[1:])
    return np.split(order, bounds[:-1])


# ---- the device solver ----------------------------------------------------------

def _maxits_int(maxits) -> int:
    if maxits is None or (isinstance(maxits, float) and math.isinf(maxits)):
        return 1 << 62
    return int(maxits)


def _options(options: dict | None) -> AcgOptions:
    """acg_options from a dict of knob names; a misspelled knob raises."""
    opts = AcgOptions()
    known = dict(AcgOptions._fields_)
    for k, v in (options or {}).items():
        if k not in known:
            raise ValueError(f"unknown solver option {k!r}; known: {sorted(known)}")
        setattr(opts, k, float(v) if known[k] is ctypes.c_double else int(v))
    return opts


class DeviceLapSolver:
    """The closure `f` of approxchol_lapGreedy (src/approxChol.jl:1624) with the
    solve on the GPU.  Holds the uploaded lap(a) and LDLinv until closed."""

    def __init__(self, a, ldli: LDLinv, *, tol=1e-6, maxits=1000, maxtime=math.inf, verbose=False, pcgIts=None,
                 params: ApproxCholParams | None = None, precision="fp64", options: dict | None = None):
        a = _csc(a)
        self.n = a.shape[0]
        self.ldli = ldli
        self.params = params or ApproxCholParams()
        self.defaults = dict(tol=tol, maxits=maxits, maxtime=maxtime, verbose=verbose, pcgIts=pcgIts,
                             precision=precision)
        opts = _options(options)
        h = ctypes.c_void_p()
        check(lib().acg_create(self.n, a.indptr.astype(np.int64), a.indices.astype(np.int64),
                               np.ascontiguousarray(a.data), ldli.col, ldli.colptr, ldli.rowval, ldli.fval, ldli.d,
                               ldli.nnz, 1, ctypes.byref(opts), ctypes.byref(h)))
        self._h = h
        self._lib = lib()
        self.last_info: list[AcgSolveInfo] = []

    def stats(self) -> dict:
        s = AcgStats()
        check(lib().acg_solver_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in AcgStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            # the library handle taken at creation: module globals may be gone
            # when this runs from __del__ at interpreter exit
            self._lib.acg_destroy(self._h)
            self._h = None

    __del__ = close

    def __call__(self, b, tol=None, maxits=None, maxtime=None, verbose=None, pcgIts=None, precision=None):
        d = self.defaults
        tol = d["tol"] if tol is None else tol
        maxits = d["maxits"] if maxits is None else maxits
        maxtime = d["maxtime"] if maxtime is None else maxtime
        verbose = d["verbose"] if verbose is None else verbose
        pcgIts = d["pcgIts"] if pcgIts is None else pcgIts
        precision = d["precision"] if precision is None else precision
        b = np.asarray(b, dtype=np.float64)
        if b.shape[0] != self.n:
            raise ValueError(f"rhs has {b.shape[0]} rows, solver has {self.n}")
        cols = b.reshape(self.n, -1)
        k = cols.shape[1]
        B = np.ascontiguousarray(cols.T)  # each right-hand side contiguous
        X = np.empty_like(B)
        infos = (AcgSolveInfo * k)()
        rc = check(lib().acg_solve(self._h, B, X, k, self.n, float(tol), _maxits_int(maxits), float(maxtime),
                                   int(self.params.stag_test), _PRECISIONS[precision], infos))
        self.last_info = list(infos)
        its = max(int(i.iterations) for i in infos) if k else 0
        if pcgIts is not None and len(pcgIts) > 0:
            pcgIts[0] = its
        if verbose:
            for i in infos:
                print(f"PCG stopped after: {i.solve_ms / 1e3:.3f} seconds and {i.iterations} iterations with relative "
                      f"error {i.relres} ({_lib.STOP_NAMES.get(i.status, i.status)}).")
        x = X.T.reshape(b.shape)
        return x

    def solve_async(self, b, tol=None, maxits=None, maxtime=None, precision=None) -> "AsyncSolve":
        """Enqueue the solve of b (n, or n x k with k <= 64) and return at once
        (acg_solve_async).  The solver runs its requests in order, overlapping
        one request's host copies with another's solve."""
        d = self.defaults
        tol = d["tol"] if tol is None else tol
        maxits = d["maxits"] if maxits is None else maxits
        maxtime = d["maxtime"] if maxtime is None else maxtime
        precision = d["precision"] if precision is None else precision
        b = np.asarray(b, dtype=np.float64)
        if b.shape[0] != self.n:
            raise ValueError(f"rhs has {b.shape[0]} rows, solver has {self.n}")
        cols = b.reshape(self.n, -1)
        B = np.ascontiguousarray(cols.T)
        X = np.empty_like(B)
        req = ctypes.c_void_p()
        check(lib().acg_solve_async(self._h, B.ctypes.data, X.ctypes.data, B.shape[0], self.n, float(tol),
                                    _maxits_int(maxits), float(maxtime), int(self.params.stag_test),
                                    _PRECISIONS[precision], ctypes.byref(req)))
        return AsyncSolve(req, B, X, b.shape)

    # one-shot device operations used by the parity tests
    def ldlsolve(self, r, precision="fp64"):
        r = np.ascontiguousarray(r, dtype=np.float64)
        y = np.empty_like(r)
        check(lib().acg_ldlsolve(self._h, r, y, _PRECISIONS[precision]))
        return y

    def time_kernels(self, precision="fp64", reps=20) -> dict:
        t = _lib.AcgKernelTimes()
        check(lib().acg_time_kernels(self._h, _PRECISIONS[precision], int(reps), ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in _lib.AcgKernelTimes._fields_}

    def time_kernels_batch(self, nrhs, precision="mixed", reps=5) -> dict:
        t = _lib.AcgKernelTimes()
        check(lib().acg_time_kernels_batch(self._h, _PRECISIONS[precision], int(nrhs), int(reps), ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in _lib.AcgKernelTimes._fields_}

    def time_sweep_levels(self, levels, nrhs=64, precision="mixed", reps=5) -> list:
        """The batched sweeps cut at each level L of `levels`: the forward sweep
        over levels 0..L and the backward sweep over levels >= L, per launch
        (ms), with the tasks each covers.  Diagnostic (acg_time_sweep_levels)."""
        lv = np.ascontiguousarray(levels, dtype=np.int32)
        m = lv.size
        f = np.zeros(m)
        b = np.zeros(m)
        tf = np.zeros(m, np.int32)
        tb = np.zeros(m, np.int32)
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        check(lib().acg_time_sweep_levels(self._h, _PRECISIONS[precision], int(nrhs), int(reps), m, ptr(lv), ptr(f),
                                          ptr(b), ptr(tf), ptr(tb)))
        return [{"level": int(lv[i]), "forward_tasks": int(tf[i]), "forward_ms": float(f[i]),
                 "backward_tasks": int(tb[i]), "backward_ms": float(b[i])} for i in range(m)]

    def lap_mul(self, x, precision="fp64"):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        check(lib().acg_lap_mul(self._h, x, y, _PRECISIONS[precision]))
        return y


class AsyncSolve:
    """A solve enqueued by DeviceLapSolver.solve_async.  Holds its right-hand
    sides and solution block until wait() (the library reads and writes them
    asynchronously)."""

    def __init__(self, req, B, X, shape):
        self._req = req
        self._B, self._X, self._shape = B, X, shape
        self._lib = lib()
        self.info: list[AcgSolveInfo] = []
        self.rc = None

    def done(self) -> bool:
        """True once the solve has finished (wait() will not block)."""
        if self._req is None:
            return True
        return check(self._lib.acg_poll(self._req)) == 1

    def wait(self):
        """Block until the solve has finished; returns x shaped like b."""
        if self._req is not None:
            k = self._X.shape[0]
            infos = (AcgSolveInfo * k)()
            req, self._req = self._req, None
            self.rc = check(self._lib.acg_wait(req, infos))
            self.info = list(infos)
        return self._X.T.reshape(self._shape)

    def __del__(self):
        if getattr(self, "_req", None) is not None:
            self._lib.acg_wait(self._req, None)
            self._req = None


class ServeLoop:
    """A device-resident serving loop on one solver (acg_serve_open): requests
    of one or more right-hand sides join the running loop as slots free up,
    and every right-hand side is its own PCG system with the reference's stop
    rules.  submit() returns a Ticket at once; Ticket.wait() gives x."""

    def __init__(self, solver: DeviceLapSolver, precision="mixed", slots=64, queue=0):
        h = ctypes.c_void_p()
        check(lib().acg_serve_open(solver._h, _PRECISIONS[precision], int(slots), int(queue), ctypes.byref(h)))
        self._h = h
        self._lib = lib()
        self.solver = solver
        self.n = solver.n
        self.precision = precision

    def submit(self, b, tol=1e-8, maxits=2000, maxtime=math.inf, stag_test=None) -> "Ticket":
        b = np.asarray(b, dtype=np.float64)
        if b.shape[0] != self.n:
            raise ValueError(f"rhs has {b.shape[0]} rows, solver has {self.n}")
        cols = b.reshape(self.n, -1)
        B = np.ascontiguousarray(cols.T)
        X = np.empty_like(B)
        t = ctypes.c_void_p()
        st = self.solver.params.stag_test if stag_test is None else stag_test
        check(self._lib.acg_serve_submit(self._h, B.ctypes.data, X.ctypes.data, B.shape[0], self.n, float(tol),
                                         _maxits_int(maxits), float(maxtime), int(st), ctypes.byref(t)))
        return Ticket(self, t, X, b.shape)

    def stats(self) -> dict:
        """Loop launches so far and right-hand sides finished."""
        la, co = ctypes.c_int64(), ctypes.c_int64()
        check(self._lib.acg_serve_stats(self._h, ctypes.byref(la), ctypes.byref(co)))
        return {"launches": la.value, "completed": co.value}

    def close(self):
        if getattr(self, "_h", None):
            check(self._lib.acg_serve_close(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Ticket:
    """A request submitted to a ServeLoop; holds its x block until wait()."""

    def __init__(self, loop, t, X, shape):
        self._loop, self._t, self._X, self._shape = loop, t, X, shape
        self.info: list[AcgSolveInfo] = []
        self.rc = None

    def done(self) -> bool:
        if self._t is None:
            return True
        return check(self._loop._lib.acg_serve_poll(self._t)) == 1

    def wait(self):
        if self._t is not None:
            k = self._X.shape[0]
            infos = (AcgSolveInfo * k)()
            t, self._t = self._t, None
            rc = self._loop._lib.acg_serve_wait(t, infos)
            self.info = list(infos)
            self.rc = check(rc)
        return self._X.T.reshape(self._shape)


class GroupSolver:
    """Many graphs solved in the same launches: the block-diagonal union of the
    graphs with the union of their factors, each graph its own PCG system
    (blockSolver's per-component solves, src/solverInterface.jl:152-188, all at
    once).  Every graph must be connected and have at least 2 vertices."""

    def __init__(self, graphs, factors=None, *, tol=1e-6, maxits=1000, maxtime=math.inf, stag_test=5,
                 precision="fp64", options: dict | None = None):
        graphs = [_csc(a) for a in graphs]
        if factors is None:
            factors = [approx_chol(a) for a in graphs]
        sizes = [a.shape[0] for a in graphs]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.n = int(self.offsets[-1])
        self.defaults = dict(tol=tol, maxits=maxits, maxtime=maxtime, precision=precision)
        self.stag_test = stag_test
        a = _csc(sp.block_diag(graphs, format="csc"))
        # union factor: columns of every graph in turn, vertex ids shifted (1-based)
        cols, ptrs, rows, fvals, ds = [], [], [], [], []
        base_entry = 0
        for f, off in zip(factors, self.offsets[:-1]):
            cols.append(f.col + off)
            ptrs.append(f.colptr[:-1] + base_entry)
            rows.append(f.rowval + off)
            fvals.append(f.fval)
            ds.append(f.d)
            base_entry += f.nnz
        col = np.concatenate(cols).astype(np.int64)
        colptr = np.concatenate(ptrs + [np.array([base_entry + 1])]).astype(np.int64)
        rowval = np.concatenate(rows).astype(np.int64)
        fval = np.concatenate(fvals)
        d = np.concatenate(ds)
        self.factor = LDLinv(col, colptr, rowval, fval, d)
        opts = _options(options)
        h = ctypes.c_void_p()
        check(lib().acg_create_group(len(graphs), self.offsets, self.n, a.indptr.astype(np.int64),
                                     a.indices.astype(np.int64), np.ascontiguousarray(a.data), col, col.shape[0],
                                     colptr, rowval, fval, d, fval.shape[0], 1, ctypes.byref(opts), ctypes.byref(h)))
        self._h = h
        self._lib = lib()
        self.ngraphs = len(graphs)
        self.last_info = []

    def __call__(self, bs, tol=None, maxits=None, maxtime=None, precision=None):
        """bs: one right-hand side per graph (list), or the union vector; returns
        the same shape.  precision "fp64" (default) or "mixed" (each graph's FP32
        PCG inside its own FP64 refinement)."""
        d = self.defaults
        tol = d["tol"] if tol is None else tol
        maxits = d["maxits"] if maxits is None else maxits
        maxtime = d["maxtime"] if maxtime is None else maxtime
        precision = d["precision"] if precision is None else precision
        as_list = isinstance(bs, (list, tuple))
        b = np.ascontiguousarray(np.concatenate(bs) if as_list else bs, dtype=np.float64)
        x = np.empty_like(b)
        infos = (AcgSolveInfo * self.ngraphs)()
        check(lib().acg_solve_group(self._h, b, x, float(tol), _maxits_int(maxits), float(maxtime), int(self.stag_test),
                                    _PRECISIONS[precision], infos))
        self.last_info = list(infos)
        if as_list:
            return [x[self.offsets[g]:self.offsets[g + 1]] for g in range(self.ngraphs)]
        return x

    def stats(self) -> dict:
        s = AcgStats()
        check(lib().acg_solver_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in AcgStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            # the library handle taken at creation: module globals may be gone
            # when this runs from __del__ at interpreter exit
            self._lib.acg_destroy(self._h)
            self._h = None

    __del__ = close


def null_solver(b, **kw):
    """`nullSolver` (src/solverInterface.jl:69-72): zeros."""
    return np.zeros_like(np.asarray(b, dtype=np.float64))


class _DenseGroundedSolver:
    """`lapWrapConnected(chol_sddm, a)` (src/solverInterface.jl:113-142) for a
    component with fewer than 50 vertices, as the reference does: drop the
    vertex of largest degree, Cholesky-solve the rest, centre the result."""

    def __init__(self, a):
        la = lap(a).toarray()
        self.N = la.shape[0]
        ind = int(np.argmax(np.diag(la)))
        self.leave = np.array([i for i in range(self.N) if i != ind], dtype=np.int64)
        sub = la[np.ix_(self.leave, self.leave)]
        self.chol = np.linalg.cholesky(sub)

    def __call__(self, b, **kw):
        b = np.asarray(b, dtype=np.float64)
        bs = b[self.leave] - b.mean()
        y = np.linalg.solve(self.chol, bs)
        xs = np.linalg.solve(self.chol.T, y)
        x = np.zeros(self.N)
        x[self.leave] = xs
        return x - x.mean()


class _GroupPart:
    """Every component with at least 50 vertices of a disconnected graph,
    solved together: one GroupSolver over their union, so each solve is one
    launch for all of them (the reference solves them one after another in
    blockSolver, src/solverInterface.jl:152-188)."""

    def __init__(self, graphs, factors, params, precision, options):
        self.precision = precision
        if len(graphs) == 1:
            # one large component: the one-graph solver (dense tail and all)
            self.group = None
            self.single = DeviceLapSolver(graphs[0], factors[0], params=params, options=options)
        else:
            self.group = GroupSolver(graphs, factors, stag_test=params.stag_test, options=options)
            self.single = None

    def __call__(self, bs, tol, maxits, maxtime, precision=None):
        precision = self.precision if precision is None else precision
        if self.single is not None:
            x = self.single(bs[0], tol=tol, maxits=maxits, maxtime=maxtime, precision=precision)
            return [x], int(self.single.last_info[0].iterations)
        xs = self.group(bs, tol=tol, maxits=maxits, maxtime=maxtime, precision=precision)
        its = max(int(i.iterations) for i in self.group.last_info)
        return xs, its


class _BlockSolver:
    """`blockSolver` (src/solverInterface.jl:152-188): the components of a
    disconnected graph solved apart and assembled.  Components of fewer than 50
    vertices (and singletons) are solved on the host as the reference does;
    the large ones share one group launch per right-hand side."""

    def __init__(self, comps, solvers, defaults, group=None, group_comps=()):
        self.comps = comps
        self.solvers = solvers
        self.defaults = defaults
        self.group = group
        self.group_comps = list(group_comps)

    def __call__(self, b, tol=None, maxits=None, maxtime=None, verbose=None, pcgIts=None, precision=None):
        d = self.defaults
        tol = d["tol"] if tol is None else tol
        maxits = d["maxits"] if maxits is None else maxits
        maxtime = d["maxtime"] if maxtime is None else maxtime
        pcgIts = d["pcgIts"] if pcgIts is None else pcgIts
        b = np.asarray(b, dtype=np.float64)
        x = np.zeros(b.shape)
        its = 0
        for ind, s in zip(self.comps, self.solvers):
            if b.ndim == 1:
                x[ind] = s(b[ind])
            else:
                for c in range(b.shape[1]):
                    x[ind, c] = s(b[ind, c])
        if self.group is not None:
            cols = b.reshape(b.shape[0], -1)
            xcols = x.reshape(b.shape[0], -1)
            for c in range(cols.shape[1]):
                xs, it = self.group([cols[ind, c] for ind in self.group_comps], tol, maxits, maxtime, precision)
                for ind, xi in zip(self.group_comps, xs):
                    xcols[ind, c] = xi
                its = max(its, it)
        if pcgIts is not None and len(pcgIts) > 0:
            pcgIts[0] = its
        return x


def approxchol_lap1(a, *, tol=1e-6, maxits=1000, maxtime=math.inf, verbose=False, pcgIts=None,
                    params: ApproxCholParams | None = None, precision="fp64", options=None):
    """Dispatch on params.order (src/approxChol.jl:1791-1851); the :deg order is
    approxchol_lapGreedy (src/approxChol.jl:1581-1626)."""
    params = params or ApproxCholParams()
    t1 = time.time()
    ldli = approx_chol(a, params)
    s = DeviceLapSolver(a, ldli, tol=tol, maxits=maxits, maxtime=maxtime, verbose=verbose, pcgIts=pcgIts,
                        params=params, precision=precision, options=options)
    if verbose:
        a = _csc(a)
        dg = np.asarray(a.sum(axis=0)).ravel()
        names = {"deg": "greedy degree", "given": "given", "wdeg": "wted degree", "random": "random"}
        print(f"Using {names.get(params.order, params.order)} ordering. Factorization time: ", time.time() - t1)
        print(f"Factorization size: {2 * ldli.nnz}")
        print("Ratio of operator edges to original edges: ", 2 * ldli.nnz / a.nnz)
        print("ratio of max to min diagonal of laplacian : ", dg.max() / dg.min())
    return s


def approxchol_lap(a, *, tol=1e-6, maxits=1000, maxtime=math.inf, verbose=False, pcgIts=None,
                   params: ApproxCholParams | None = None, precision="fp64", options=None):
    """`approxchol_lap` (src/approxChol.jl:1522-1545) through `lapWrapComponents`
    (src/solverInterface.jl:212-275)."""
    a = _csc(a)
    if a.nnz and a.data.min() < 0:
        raise ValueError("Adjacency matrix can not have negative edge weights")
    if a.diagonal().any():
        import warnings
        warnings.warn("The matrix should not have any nonzero diagonal entries.")
        a = _csc(a - sp.diags(a.diagonal()))
        a.eliminate_zeros()
    kw = dict(tol=tol, maxits=maxits, maxtime=maxtime, verbose=verbose, pcgIts=pcgIts, params=params,
              precision=precision, options=options)
    co = components(a)
    if co.max() == 1:
        return approxchol_lap1(a, **kw)
    comps = vec_to_comps(co)
    host_comps, solvers, big = [], [], []
    sizes = np.array([len(c) for c in comps])
    null_idx = np.where(sizes == 1)[0]
    if null_idx.size:
        host_comps.append(np.concatenate([comps[i] for i in null_idx]))
        solvers.append(null_solver)
    for i, ind in enumerate(comps):
        if sizes[i] == 1:
            continue
        if len(ind) < 50:
            host_comps.append(ind)
            solvers.append(_DenseGroundedSolver(a[ind][:, ind]))
        else:
            big.append(ind)
    group = None
    params = params or ApproxCholParams()
    if big:
        graphs = [_csc(a[ind][:, ind]) for ind in big]
        t1 = time.time()
        factors = [approx_chol(g, params) for g in graphs]
        if verbose:
            print(f"Factorization time for {len(big)} components: ", time.time() - t1)
        group = _GroupPart(graphs, factors, params, precision, options)
    return _BlockSolver(host_comps, solvers, dict(tol=tol, maxits=maxits, maxtime=maxtime, verbose=verbose,
                                                  pcgIts=pcgIts), group=group, group_comps=big)


def approxchol_lap2(a, *, tol=1e-6, maxits=1000, maxtime=math.inf, verbose=False, pcgIts=None,
                    params: ApproxCholParams | None = None, precision="fp64", options=None):
    """`approxchol_lap2` (src/approxChol.jl:1559-1578): approxchol_lap with the
    split/merge elimination, ApproxCholParams(:deg, stag_test, 2, 2)."""
    st = (params or ApproxCholParams()).stag_test
    return approxchol_lap(a, tol=tol, maxits=maxits, maxtime=maxtime, verbose=verbose, pcgIts=pcgIts,
                          params=ApproxCholParams("deg", st, 2, 2), precision=precision, options=options)


def adj_val_and_excess(sddm):
    """`adjValAndExcess` (src/graphOps.jl:43-48): the adjacency a = diag(M) - M
    (off-diagonal weights, no stored diagonal), the diagonal, and the row sums
    M*1 (the diagonal's excess over the off-diagonal weights)."""
    m = _csc(sddm)
    dval = np.asarray(m.diagonal(), dtype=np.float64)
    a = _csc(sp.diags(dval) - m)
    a.setdiag(0.0)
    a.eliminate_zeros()
    a = _csc(a)
    dexcess = np.asarray(m @ np.ones(m.shape[0]), dtype=np.float64)
    return a, dval, dexcess


def extend_matrix(a, dval, dexcess):
    """`extendMatrix` (src/graphOps.jl:56-79): append a ground vertex joined to
    every vertex whose excess exceeds 100*eps times its diagonal, with the
    excess as the edge weight; `a` itself when there is no excess at all."""
    if np.abs(dexcess).sum() == 0:
        return a
    pos = np.where(dexcess > 100 * np.finfo(np.float64).eps * dval)[0]
    n = a.shape[0]
    coo = a.tocoo()
    i = np.concatenate([coo.row, pos, np.full(pos.size, n)])
    j = np.concatenate([coo.col, np.full(pos.size, n), pos])
    v = np.concatenate([coo.data, dexcess[pos], dexcess[pos]])
    return _csc(sp.csc_matrix((v, (i, j)), shape=(n + 1, n + 1)))


def approxchol_sddm(sddm, *, tol=1e-6, maxits=1000, maxtime=math.inf, verbose=False, pcgIts=None,
                    params: ApproxCholParams | None = None, precision="fp64", options=None):
    """`approxchol_sddm = sddmWrapLap(approxchol_lap)` (src/approxChol.jl:1862,
    src/solverInterface.jl:324-350): solves M x = b for a symmetric, diagonally
    dominant M with non-positive off-diagonals by grounding the diagonal excess
    in one extra vertex and solving the extended Laplacian system on the GPU."""
    m = _csc(sddm)
    if m.shape[0] != m.shape[1]:
        raise ValueError("the SDDM matrix must be square")
    n = m.shape[0]
    a, dval, dexcess = adj_val_and_excess(m)
    a1 = extend_matrix(a, dval, dexcess)
    kw = dict(tol=tol, maxits=maxits, maxtime=maxtime, verbose=verbose, pcgIts=pcgIts, params=params,
              precision=precision, options=options)
    if a1.shape == m.shape:
        # no excess: the matrix is a Laplacian (src/solverInterface.jl:338-341)
        return approxchol_lap(a, **kw)
    F = approxchol_lap(a1, **kw)
    defaults = dict(tol=tol, maxits=maxits, maxtime=maxtime, verbose=verbose, pcgIts=pcgIts)

    def f(b, tol=None, maxits=None, maxtime=None, verbose=None, pcgIts=None):
        b = np.asarray(b, dtype=np.float64)
        if b.shape[0] != n:
            raise ValueError(f"rhs has {b.shape[0]} rows, matrix has {n}")
        call = {k: (v if v is not None else defaults[k]) for k, v in
                dict(tol=tol, maxits=maxits, maxtime=maxtime, verbose=verbose, pcgIts=pcgIts).items()}
        xaug = F(np.concatenate([b, [-b.sum()]]), **call)
        xaug = xaug - xaug[-1]
        return xaug[:n]

    f.solver = F
    return f


_seed_from_entropy_done = False


def _init():
    global _seed_from_entropy_done
    if not _seed_from_entropy_done:
        try:
            _seed_from_entropy()
        except ImportError:
            pass
        _seed_from_entropy_done = True
