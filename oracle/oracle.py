"""ORACLE — test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker (or, for the CPU baseline, as the timed
restatement of the reference's CPU solve).  The product never imports it.

Wraps liboracle.so, the plain-C restatement of the reference's solve phase
(acg_oracle.c: lap, SparseArrays mat-vec, LDLsolver/forward!/backward!, pcg,
the closure f), and adds an exact solve of the grounded Laplacian with
SuperLU (scipy) as an independent reference for x.
"""
from __future__ import annotations

import ctypes
import subprocess
import sys
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
SRC = HERE / "acg_oracle.c"
LIB = HERE / "liboracle.so"
if str(HERE) not in sys.path:
    sys.path.insert(0, str(HERE))

i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


class _Problem(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("l_colptr", ctypes.c_void_p), ("l_rowval", ctypes.c_void_p),
                ("l_nzval", ctypes.c_void_p), ("col", ctypes.c_void_p), ("colptr", ctypes.c_void_p),
                ("rowval", ctypes.c_void_p), ("fval", ctypes.c_void_p), ("d", ctypes.c_void_p)]


def build(force: bool = False) -> Path:
    """Compile liboracle.so with gcc (no FMA contraction, like Julia)."""
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["gcc", "-O3", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", str(SRC), "-o", str(tmp),
                    "-lm"], check=True)
    tmp.replace(LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        L.oracle_lap_nnz.restype = ctypes.c_int64
        L.oracle_lap_nnz.argtypes = [ctypes.c_int64, i64p]
        L.oracle_lap.restype = None
        L.oracle_lap.argtypes = [ctypes.c_int64, i64p, i64p, f64p, i64p, i64p, f64p]
        L.oracle_spmv.restype = None
        L.oracle_spmv.argtypes = [ctypes.c_int64, i64p, i64p, f64p, f64p, f64p]
        L.oracle_ldlsolve.restype = None
        L.oracle_ldlsolve.argtypes = [ctypes.c_int64, i64p, i64p, i64p, f64p, f64p, f64p, f64p]
        L.oracle_forward.restype = None
        L.oracle_forward.argtypes = [ctypes.c_int64, i64p, i64p, i64p, f64p, f64p]
        L.oracle_backward.restype = None
        L.oracle_backward.argtypes = [ctypes.c_int64, i64p, i64p, i64p, f64p, f64p]
        for fn in (L.oracle_pcg, L.oracle_solve):
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.POINTER(_Problem), f64p, f64p, ctypes.c_double, ctypes.c_int64, ctypes.c_double,
                           ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)]
        _lib = L
    return _lib


def _julia_csc(a):
    a = sp.csc_matrix(a, dtype=np.float64)
    a.sum_duplicates()
    a.sort_indices()
    return a.indptr.astype(np.int64) + 1, a.indices.astype(np.int64) + 1, np.ascontiguousarray(a.data)


class OracleLap:
    """lap(a) in Julia's CSC layout, with the reference's mat-vec."""

    def __init__(self, a):
        cp, rv, nz = _julia_csc(a)
        n = cp.shape[0] - 1
        L = lib()
        nnz = L.oracle_lap_nnz(n, cp)
        self.n = n
        self.colptr = np.empty(n + 1, np.int64)
        self.rowval = np.empty(nnz, np.int64)
        self.nzval = np.empty(nnz, np.float64)
        L.oracle_lap(n, cp, rv, nz, self.colptr, self.rowval, self.nzval)

    def mul(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        q = np.empty_like(p)
        lib().oracle_spmv(self.n, self.colptr, self.rowval, self.nzval, p, q)
        return q

    def scipy(self):
        return sp.csc_matrix((self.nzval, self.rowval - 1, self.colptr - 1), shape=(self.n, self.n))


def ldlsolve(ldli, b):
    """y = LDLsolver(ldli, b) (src/approxChol.jl:1347-1366)."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    y = np.empty_like(b)
    lib().oracle_ldlsolve(b.shape[0], ldli.col, ldli.colptr, ldli.rowval, ldli.fval, ldli.d, b, y)
    return y


class OracleSolver:
    """The closure f(b) of src/approxChol.jl:1624 on the CPU (FP64)."""

    def __init__(self, a, ldli, stag_test=5):
        self.lap = OracleLap(a)
        self.ldli = ldli
        self.stag_test = stag_test
        self._keep = (self.lap.colptr, self.lap.rowval, self.lap.nzval, ldli.col, ldli.colptr, ldli.rowval,
                      ldli.fval, ldli.d)
        self.prob = _Problem(self.lap.n, *[x.ctypes.data for x in self._keep])

    def __call__(self, b, tol=1e-6, maxits=1000, maxtime=float("inf"), center=True):
        """Returns (x, iterations, stop code, final recursive |r|/|b|)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty_like(b)
        its = ctypes.c_int64()
        nr = ctypes.c_double()
        fn = lib().oracle_solve if center else lib().oracle_pcg
        mi = (1 << 62) if maxits == float("inf") else int(maxits)
        rc = fn(ctypes.byref(self.prob), b, x, tol, mi, maxtime, self.stag_test, ctypes.byref(its), ctypes.byref(nr))
        return x, its.value, rc, nr.value


def _magnitude_second(ev, upper):
    """The reference's lower eigenvalue: upper minus the second-largest
    magnitude eigenvalue of upper*I - G (src/approxChol.jl:1931-1933)."""
    shifted = upper - ev
    order = np.argsort(-np.abs(shifted), kind="stable")
    return upper - shifted[order[1]]


def cond_number(a, ldli):
    """condNumber(a, ldli) (src/approxChol.jl:1880-1936): upper/lower of the
    operator g(b) = D^-1/2 forward!(lap(a) * backward!(D^-1/2 b)), entries with
    d = 0 zeroed.  The reference estimates the two eigenvalues with ARPACK's
    eigs at tol 1e-2; here g is formed densely (n up to a few thousand) and its
    eigenvalues are exact, with the same choice of upper and lower: upper is
    the largest, lower = upper minus the second-largest magnitude of upper - g."""
    n = ldli.n
    L = OracleLap(a)
    d = np.asarray(ldli.d, dtype=np.float64)
    dis = np.where(d != 0, 1.0 / np.sqrt(np.where(d != 0, d, 1.0)), 0.0)
    lib_ = lib()
    g = np.empty((n, n))
    for j in range(n):
        y = np.zeros(n)
        y[j] = dis[j]
        lib_.oracle_backward(n, ldli.col, ldli.colptr, ldli.rowval, ldli.fval, y)
        y = np.ascontiguousarray(L.mul(y))
        lib_.oracle_forward(n, ldli.col, ldli.colptr, ldli.rowval, ldli.fval, y)
        g[:, j] = y * dis
    ev = np.linalg.eigvalsh(0.5 * (g + g.T))
    upper = float(ev[-1])
    return upper / float(_magnitude_second(ev, upper))


def cond_number_of_operator(m):
    """The same upper/lower for a dense operator m = P lap(a) given column by
    column (P a preconditioner applied on a device): its eigenvalues are those
    of g up to rounding (P L and D^-1/2 U' L U D^-1/2 share their nonzero
    eigenvalues), so the two condition numbers agree."""
    ev = np.sort(np.linalg.eigvals(np.asarray(m, dtype=np.float64)).real)
    upper = float(ev[-1])
    return upper / float(_magnitude_second(ev, upper))


def exact_solve(a, b):
    """x with lap(a) x = b - mean(b) on a connected graph, by SuperLU on the
    Laplacian grounded at its vertex of largest degree, then centred."""
    from scipy.sparse.linalg import splu
    a = sp.csc_matrix(a, dtype=np.float64)
    la = (sp.diags(np.asarray(a.sum(axis=1)).ravel()) - a).tocsc()
    n = la.shape[0]
    ind = int(np.argmax(la.diagonal()))
    keep = np.r_[0:ind, ind + 1:n]
    sub = la[keep][:, keep].tocsc()
    bb = np.asarray(b, dtype=np.float64)
    bb = bb - bb.mean()
    x = np.zeros(n)
    x[keep] = splu(sub).solve(bb[keep])
    return x - x.mean()


def relres(a, x, b):
    """|lap(a) x - b| / |b| as src/compare_solvers.jl:138 measures it."""
    a = sp.csc_matrix(a, dtype=np.float64)
    la = sp.diags(np.asarray(a.sum(axis=1)).ravel()) - a
    return float(np.linalg.norm(la @ x - b) / np.linalg.norm(b))


def center(x):
    x = np.asarray(x, dtype=np.float64)
    return x - x.mean()
