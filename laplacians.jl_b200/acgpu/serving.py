"""Continuous-batching solve server on one GPU.

Requests name a registered graph and carry one or more right-hand sides.
Every graph that has work is resident on the device: its solver (lap(a) and
the LDLinv factor, uploaded once) and a device-resident serving loop
(ServeLoop, acg_serve_* in include/acgpu.h) whose slots are the batched
solver's columns.  A request's right-hand sides are handed to the loop as
soon as they arrive; the loop admits them into free slots between PCG
iterations while other solves are running, and hands each solve back the
moment it stops.  So requests that arrive while others are on the GPU join
the running launch, and nothing waits for a batch to fill or to drain.

Residency is bounded by an HBM budget: a graph is uploaded when its first
request arrives (outside the server's lock, so requests on resident graphs
are not held up), and when the budget would be exceeded the least recently
used graphs with no work in flight are evicted.  Different graphs have their
own loops on their own CUDA streams; their kernels interleave on the device.

Every right-hand side stays its own PCG system, so a result is that of the
same request solved alone up to rounding (tests/test_gpu_serve_loop.py and
tests/test_gpu_serving.py hold it to the batched tests' tolerances).

The reference has no server: its closure solves one vector per call
(src/approxChol.jl:1624); this module is the serving layer around it.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from .solvers import (DeviceLapSolver, ServeLoop, _csc, _DenseGroundedSolver, approx_chol, components,
                      seed as rng_seed, vec_to_comps)

__all__ = ["SolveServer", "Request", "AdmissionError"]


class AdmissionError(RuntimeError):
    """A graph whose solver alone exceeds the server's HBM budget."""


@dataclass(eq=False)  # compared by identity: the fields hold numpy arrays
class Request:
    gid: object
    B: np.ndarray          # n x k right-hand sides (k >= 1)
    tol: float
    t_submit: float
    future: Future = field(default_factory=Future)
    t_start: float = 0.0
    t_done: float = 0.0
    ticket: object = None
    internal: bool = False  # one component's part of a request on a disconnected graph


class _GraphEntry:
    def __init__(self, gid, a, ldli):
        self.gid = gid
        self.a = a
        self.ldli = ldli
        self.solver: DeviceLapSolver | None = None
        self.loop: ServeLoop | None = None
        self.bytes = 0
        self.loading = False
        self.inflight = 0
        self.last_used = 0.0
        self.queue: collections.deque[Request] = collections.deque()


class _Composite:
    """A disconnected graph (lapWrapComponents, src/solverInterface.jl:212-275):
    components of at least 50 vertices are graphs of their own in the server
    (keys (gid, k)), smaller ones are solved on the host, singletons get 0."""

    def __init__(self, n, big, small):
        self.n = n
        self.big = big        # [(index array, sub-gid)]
        self.small = small    # [(index array, host solver)]


class SolveServer:
    """Serve Laplacian solves with device-resident factors and continuous batching.

    hbm_budget: bytes of device memory the resident graphs may hold together.
    precision: "mixed" (FP32 PCG in FP64 refinement) or "fp64".
    slots: columns of each graph's serving loop (8, 16, 32 or 64).
    queue: requests that may wait in a loop's ring beside its busy slots.
    unbatched: the baseline instead: one request at a time, one right-hand
      side per solve, through the plain solve entry.
    """

    def __init__(self, hbm_budget: int, slots: int = 64, precision: str = "mixed", maxits: int = 2000,
                 unbatched: bool = False, queue: int = 64):
        self.unbatched = bool(unbatched)
        self.hbm_budget = int(hbm_budget)
        self.slots = int(slots)
        self.queue = int(queue)
        self.precision = precision
        self.maxits = maxits
        self._graphs: dict[object, _GraphEntry] = {}
        self._cv = threading.Condition()
        self._stop = False
        self._resident = 0
        self._threads: list[threading.Thread] = []
        self._pending: list[Request] = []  # handed to a loop, not yet finished
        self._composites: dict[object, _Composite] = {}
        self.completed: list[Request] = []
        self.uploads = 0

    # ---- graphs -------------------------------------------------------------
    def register(self, gid, a, ldli=None, seed: int | None = None):
        """Add a graph (host factor built now, device upload on first use).  A
        disconnected graph is split into its components, as approxchol_lap does;
        its factor is then built here per component (ldli must be None)."""
        a = _csc(a)
        if seed is not None and ldli is None:
            rng_seed(seed)
        co = components(a)
        if co.max() > 1:
            if ldli is not None:
                raise ValueError("a disconnected graph is factored per component: pass ldli=None")
            big, small = [], []
            for k, ind in enumerate(vec_to_comps(co)):
                if len(ind) == 1:
                    continue
                sub = _csc(a[ind][:, ind])
                if len(ind) < 50:
                    small.append((ind, _DenseGroundedSolver(sub)))
                else:
                    big.append((ind, (gid, k)))
                    with self._cv:
                        self._graphs[(gid, k)] = _GraphEntry((gid, k), sub, approx_chol(sub))
            with self._cv:
                self._composites[gid] = _Composite(a.shape[0], big, small)
            return
        if ldli is None:
            ldli = approx_chol(a)
        with self._cv:
            self._graphs[gid] = _GraphEntry(gid, a, ldli)

    def _estimate_bytes(self, e: _GraphEntry) -> int:
        n = e.a.shape[0]
        nnz_l = e.a.nnz + n
        F = e.ldli.nnz
        structure = nnz_l * 16 + 2 * F * 16 + n * 64
        vectors = n * 8 * 30
        batch = n * self.slots * (9 * 8 + 3 * 8 + 8 * 4)
        staging = 0 if self.unbatched else n * 8 * 2 * (self.slots + self.queue)
        return int(structure + vectors + batch + staging)

    def _reserve(self, e: _GraphEntry) -> bool:
        """With the lock held: reserve e's bytes, evicting idle graphs (least
        recently used first).  False when it cannot fit now."""
        est = self._estimate_bytes(e)
        if est > self.hbm_budget:
            raise AdmissionError(f"graph {e.gid!r} needs ~{est} bytes, budget {self.hbm_budget}")
        if self._resident + est > self.hbm_budget:
            idle = [g for g in self._graphs.values()
                    if g.solver is not None and not g.loading and g.inflight == 0 and not g.queue and g is not e]
            idle.sort(key=lambda g: g.last_used)
            if self._resident - sum(g.bytes for g in idle) + est > self.hbm_budget:
                return False
            for victim in idle:
                if self._resident + est <= self.hbm_budget:
                    break
                self._evict(victim)
        e.bytes = est
        self._resident += est
        return True

    def _evict(self, g: _GraphEntry):
        if g.loop is not None:
            g.loop.close()
            g.loop = None
        g.solver.close()
        g.solver = None
        self._resident -= g.bytes
        g.bytes = 0

    def _load(self, e: _GraphEntry):
        """Upload e outside the lock; its queued requests go out afterwards."""
        err = None
        solver = loop = None
        try:
            solver = DeviceLapSolver(e.a, e.ldli)
            if not self.unbatched:
                loop = ServeLoop(solver, precision=self.precision, slots=self.slots, queue=self.queue)
        except Exception as exc:  # noqa: BLE001 - forwarded to the waiting callers
            err = exc
        with self._cv:
            e.loading = False
            if err is not None:
                self._resident -= e.bytes
                e.bytes = 0
                while e.queue:
                    e.queue.popleft().future.set_exception(err)
            else:
                e.solver, e.loop = solver, loop
                self.uploads += 1
            self._cv.notify_all()

    # ---- requests -----------------------------------------------------------
    def submit(self, gid, B, tol: float = 1e-8) -> Future:
        B = np.asarray(B, dtype=np.float64)
        if B.ndim == 1:
            B = B[:, None]
        if gid in self._composites:
            return self._submit_composite(gid, self._composites[gid], B, tol)
        return self._submit_one(gid, B, tol).future

    def _submit_one(self, gid, B, tol, internal=False) -> Request:
        req = Request(gid, B, tol, time.perf_counter(), internal=internal)
        with self._cv:
            if gid not in self._graphs:
                raise KeyError(f"graph {gid!r} not registered")
            self._graphs[gid].queue.append(req)
            self._cv.notify_all()
        return req

    def _submit_composite(self, gid, comp: _Composite, B, tol) -> Future:
        """One request on a disconnected graph: each large component's rows go
        to that component's loop; the result is assembled when all are back."""
        top = Request(gid, B, tol, time.perf_counter())
        parts = [(ind, self._submit_one(sub, np.ascontiguousarray(B[ind]), tol, internal=True))
                 for ind, sub in comp.big]
        X = np.zeros(B.shape)
        for ind, solver in comp.small:
            for c in range(B.shape[1]):
                X[ind, c] = solver(B[ind, c])
        left = [len(parts)]
        lock = threading.Lock()

        def one_done(_):
            with lock:
                left[0] -= 1
                if left[0]:
                    return
            infos, exc = [], None
            for ind, r in parts:
                try:
                    Xi, inf = r.future.result()
                    X[ind] = Xi
                    infos.append(inf)
                except Exception as e:  # noqa: BLE001
                    exc = e
            top.t_done = time.perf_counter()
            with self._cv:
                self.completed.append(top)
            if exc is not None:
                top.future.set_exception(exc)
            else:
                # per column: the component with the most iterations
                cols = [max((inf[c] for inf in infos), key=lambda i: i.iterations) for c in range(B.shape[1])]
                top.future.set_result((X, cols))

        if not parts:
            top.t_done = time.perf_counter()
            with self._cv:
                self.completed.append(top)
            top.future.set_result((X, []))
        for _, r in parts:
            r.future.add_done_callback(one_done)
        return top.future

    # ---- threads ------------------------------------------------------------
    def start(self):
        self._stop = False
        targets = [self._dispatch_unbatched] if self.unbatched else [self._dispatch, self._complete]
        for f in targets:
            t = threading.Thread(target=f, name=f"acgpu-{f.__name__}", daemon=True)
            t.start()
            self._threads.append(t)
        return self

    def stop(self, wait: bool = True):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        if wait:
            for t in self._threads:
                t.join()
        self._threads.clear()

    def close(self):
        self.stop()
        for e in self._graphs.values():
            if e.solver is not None:
                self._evict(e)
        self._resident = 0

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.close()

    def _nothing_queued(self):
        return not any(e.queue or e.loading for e in self._graphs.values())

    def _idle(self):
        return self._nothing_queued() and not self._pending

    def _dispatch(self):
        """Hand queued requests to their graphs' loops, uploading graphs as needed."""
        while True:
            load = None
            with self._cv:
                while True:
                    # in-flight solves are the completer's: it alone waits for them
                    if self._stop and self._nothing_queued():
                        return
                    ready = [e for e in self._graphs.values() if e.queue and e.loop is not None]
                    waiting = [e for e in self._graphs.values() if e.queue and e.solver is None and not e.loading]
                    if ready or waiting:
                        break
                    self._cv.wait(timeout=0.05)
                for e in ready:
                    while e.queue:
                        r = e.queue.popleft()
                        r.t_start = time.perf_counter()
                        try:
                            r.ticket = e.loop.submit(r.B, tol=r.tol, maxits=self.maxits)
                        except Exception as exc:  # noqa: BLE001
                            r.future.set_exception(exc)
                            continue
                        e.inflight += 1
                        self._pending.append(r)
                        self._cv.notify_all()
                waiting.sort(key=lambda e: e.queue[0].t_submit)
                for e in waiting:
                    try:
                        if self._reserve(e):
                            e.loading = True
                            load = e
                            break
                    except AdmissionError as exc:
                        while e.queue:
                            e.queue.popleft().future.set_exception(exc)
                if load is None and not ready:
                    # nothing fits until resident graphs finish their work
                    self._cv.wait(timeout=0.01)
            if load is not None:
                self._load(load)

    def _complete(self):
        """Finish the requests whose solves have all stopped."""
        while True:
            with self._cv:
                while not self._pending:
                    if self._stop and self._idle():
                        return
                    self._cv.wait(timeout=0.05)
                pending = list(self._pending)
            finished = []
            for r in pending:
                try:
                    if r.ticket.done():
                        finished.append(r)
                except Exception:  # noqa: BLE001 - a failed loop: wait() below raises it to the caller
                    finished.append(r)
            if not finished:
                time.sleep(5e-5)
                continue
            for r in finished:
                try:
                    X = r.ticket.wait()
                    res, exc = (X.reshape(r.B.shape).copy(), list(r.ticket.info)), None
                except Exception as e:  # noqa: BLE001
                    res, exc = None, e
                r.t_done = time.perf_counter()
                with self._cv:
                    self._pending.remove(r)
                    g = self._graphs[r.gid]
                    g.inflight -= 1
                    g.last_used = r.t_done
                    self.completed.append(r)
                    self._cv.notify_all()
                if exc is None:
                    r.future.set_result(res)
                else:
                    r.future.set_exception(exc)

    def _dispatch_unbatched(self):
        """The baseline: requests one at a time in arrival order, one right-hand
        side per solve."""
        while True:
            with self._cv:
                while True:
                    cands = [e for e in self._graphs.values() if e.queue]
                    if cands:
                        break
                    if self._stop:
                        return
                    self._cv.wait(timeout=0.05)
                e = min(cands, key=lambda g: g.queue[0].t_submit)
                r = e.queue.popleft()
                if e.solver is None:
                    try:
                        fits = self._reserve(e)
                        if not fits:  # nothing runs meanwhile: every other graph is idle
                            for g in self._graphs.values():
                                if g.solver is not None and g is not e:
                                    self._evict(g)
                            fits = self._reserve(e)
                    except AdmissionError as exc:
                        r.future.set_exception(exc)
                        continue
                    e.loading = fits
            if e.loading:
                self._load(e)
            r.t_start = time.perf_counter()
            try:
                cols, infos = [], []
                for c in range(r.B.shape[1]):
                    cols.append(e.solver(r.B[:, c], tol=r.tol, maxits=self.maxits, precision=self.precision))
                    infos += list(e.solver.last_info)
                res, exc = (np.stack(cols, axis=1), infos), None
            except Exception as ex:  # noqa: BLE001
                res, exc = None, ex
            r.t_done = time.perf_counter()
            with self._cv:
                e.last_used = r.t_done
                self.completed.append(r)
            if exc is None:
                r.future.set_result(res)
            else:
                r.future.set_exception(exc)

    # ---- statistics -------------------------------------------------------------
    def latency_stats(self):
        done = [r for r in self.completed if not r.internal]
        lat = np.array([r.t_done - r.t_submit for r in done])
        cols = sum(r.B.shape[1] for r in done)
        if not len(lat):
            return {}
        span = max(r.t_done for r in done) - min(r.t_submit for r in done)
        launches = sum(e.loop.stats()["launches"] for e in self._graphs.values() if e.loop is not None)
        return {"requests": len(lat), "solves": cols, "solves_per_s": cols / span if span > 0 else None,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3), "loop_launches": launches, "uploads": self.uploads}
