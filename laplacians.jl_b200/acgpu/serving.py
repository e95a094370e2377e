"""Continuous-batching solve server on one GPU.

Requests name a registered graph and carry 1..64 right-hand sides.  The
server keeps one device solver per graph (factor uploaded once, cached on the
device, evicted least-recently-used when a new graph would exceed the HBM
budget), a queue of pending requests per graph, and `slots` worker threads.
A free worker takes the graph whose oldest pending request is oldest, merges
that graph's pending requests (up to 64 right-hand sides) into one batched
launch on that solver's own CUDA stream, and completes their futures.  Work
of different graphs therefore overlaps on the device, and requests that
arrive while a graph's launch is running join its next launch.

Every right-hand side stays its own PCG system inside a batch, so a result is
the same as the request solved alone up to the rounding of the per-column
reductions (the batched tests bound the difference).

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

from .solvers import DeviceLapSolver, approx_chol, seed as rng_seed

__all__ = ["SolveServer", "Request", "AdmissionError"]


class AdmissionError(RuntimeError):
    """A graph whose solver alone exceeds the server's HBM budget."""


@dataclass
class Request:
    gid: object
    B: np.ndarray          # n x k right-hand sides (k >= 1)
    tol: float
    t_submit: float
    future: Future = field(default_factory=Future)
    t_start: float = 0.0
    t_done: float = 0.0


class _GraphEntry:
    def __init__(self, gid, a, ldli):
        self.gid = gid
        self.a = a
        self.ldli = ldli
        self.solver: DeviceLapSolver | None = None
        self.bytes = 0
        self.busy = False
        self.last_used = 0.0
        self.queue: collections.deque[Request] = collections.deque()


class SolveServer:
    """Serve Laplacian solves with device-resident factors and continuous batching.

    hbm_budget: bytes of device memory the cached solvers may hold together.
    slots: concurrent launches (worker threads, one CUDA stream per solver).
    precision: "mixed" (FP32 PCG in FP64 refinement) or "fp64".
    """

    def __init__(self, hbm_budget: int, slots: int = 4, precision: str = "mixed", max_batch: int = 64,
                 maxits: int = 2000, unbatched: bool = False):
        self.unbatched = bool(unbatched)  # baseline: one request per launch, one right-hand side per solve
        self.hbm_budget = int(hbm_budget)
        self.slots = int(slots)
        self.precision = precision
        self.max_batch = int(max_batch)
        self.maxits = maxits
        self._graphs: dict[object, _GraphEntry] = {}
        self._cv = threading.Condition()
        self._stop = False
        self._resident = 0
        self._workers: list[threading.Thread] = []
        self.completed: list[Request] = []
        self.launches = 0

    # ---- graphs -------------------------------------------------------------
    def register(self, gid, a, ldli=None, seed: int | None = None):
        """Add a graph (host factor built now, device upload on first use)."""
        if ldli is None:
            if seed is not None:
                rng_seed(seed)
            ldli = approx_chol(a)
        with self._cv:
            self._graphs[gid] = _GraphEntry(gid, a, ldli)

    def _ensure_resident(self, e: _GraphEntry) -> bool:
        """Called with the lock held.  Uploads e's solver if it is not on the
        device, evicting idle solvers (least recently used first, those with
        no queued work before those with some).  False when it cannot fit now
        because the other solvers are busy."""
        if e.solver is not None:
            return True
        est = self._estimate_bytes(e)
        if est > self.hbm_budget:
            raise AdmissionError(f"graph {e.gid!r} needs ~{est} bytes, budget {self.hbm_budget}")
        if self._resident + est > self.hbm_budget:
            idle = [g for g in self._graphs.values() if g.solver is not None and not g.busy and g is not e]
            idle.sort(key=lambda g: (len(g.queue) > 0, g.last_used))
            freeable = sum(g.bytes for g in idle)
            if self._resident - freeable + est > self.hbm_budget:
                return False
            for victim in idle:
                if self._resident + est <= self.hbm_budget:
                    break
                victim.solver.close()
                victim.solver = None
                self._resident -= victim.bytes
                victim.bytes = 0
        e.solver = DeviceLapSolver(e.a, e.ldli)
        e.bytes = est
        self._resident += est
        return True

    def _estimate_bytes(self, e: _GraphEntry) -> int:
        n = e.a.shape[0]
        nnz_l = e.a.nnz + n
        F = e.ldli.nnz
        structure = nnz_l * 16 + 2 * F * 16 + n * 64
        vectors = n * 8 * 30
        batch = n * self.max_batch * (9 * 8 + 3 * 8 + 8 * 4)
        return int(structure + vectors + batch)

    # ---- requests -----------------------------------------------------------
    def submit(self, gid, B, tol: float = 1e-8) -> Future:
        B = np.asarray(B, dtype=np.float64)
        if B.ndim == 1:
            B = B[:, None]
        req = Request(gid, B, tol, time.perf_counter())
        with self._cv:
            if gid not in self._graphs:
                raise KeyError(f"graph {gid!r} not registered")
            if B.shape[1] > self.max_batch:
                raise ValueError(f"at most {self.max_batch} right-hand sides per request")
            self._graphs[gid].queue.append(req)
            self._cv.notify()
        return req.future

    # ---- workers ------------------------------------------------------------
    def start(self):
        self._stop = False
        for i in range(self.slots):
            t = threading.Thread(target=self._worker, name=f"acgpu-slot-{i}", daemon=True)
            t.start()
            self._workers.append(t)
        return self

    def stop(self, wait: bool = True):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        if wait:
            for t in self._workers:
                t.join()
        self._workers.clear()

    def close(self):
        self.stop()
        for e in self._graphs.values():
            if e.solver is not None:
                e.solver.close()
                e.solver = None
        self._resident = 0

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.close()

    def _next_batch(self):
        """With the lock held: pick a graph and the requests of its next launch.
        Graphs are tried in order of their oldest pending request; one that
        cannot be made resident now is skipped for a resident one."""
        cands = [e for e in self._graphs.values() if not e.busy and e.queue]
        cands.sort(key=lambda e: e.queue[0].t_submit)
        for best in cands:
            try:
                if not self._ensure_resident(best):
                    continue
            except AdmissionError as exc:
                while best.queue:
                    best.queue.popleft().future.set_exception(exc)
                continue
            reqs, cols = [], 0
            while best.queue and cols + best.queue[0].B.shape[1] <= self.max_batch:
                r = best.queue.popleft()
                reqs.append(r)
                cols += r.B.shape[1]
                if self.unbatched:
                    break
            best.busy = True
            return best, reqs
        return None, None

    def _worker(self):
        while True:
            with self._cv:
                while True:
                    if self._stop:
                        return
                    e, reqs = self._next_batch()
                    if e is not None:
                        break
                    self._cv.wait(timeout=0.05)
            try:
                self._run(e, reqs)
            finally:
                with self._cv:
                    e.busy = False
                    e.last_used = time.perf_counter()
                    self._cv.notify_all()

    def _run(self, e: _GraphEntry, reqs: list[Request]):
        t0 = time.perf_counter()
        B = np.concatenate([r.B for r in reqs], axis=1)
        tol = min(r.tol for r in reqs)
        try:
            if self.unbatched:
                cols, infos = [], []
                for c in range(B.shape[1]):
                    cols.append(e.solver(B[:, c], tol=tol, maxits=self.maxits, precision=self.precision))
                    infos += list(e.solver.last_info)
                X = np.stack(cols, axis=1)
            else:
                X = e.solver(B, tol=tol, maxits=self.maxits, precision=self.precision)
                infos = list(e.solver.last_info)
        except Exception as exc:  # noqa: BLE001 - forwarded to every waiting caller
            for r in reqs:
                r.future.set_exception(exc)
            return
        X = X.reshape(B.shape)
        t1 = time.perf_counter()
        c = 0
        with self._cv:
            self.launches += 1
        for r in reqs:
            k = r.B.shape[1]
            r.t_start, r.t_done = t0, t1
            r.future.set_result((X[:, c:c + k].copy(), infos[c:c + k]))
            c += k
            with self._cv:
                self.completed.append(r)

    # ---- statistics -------------------------------------------------------------
    def latency_stats(self):
        lat = np.array([r.t_done - r.t_submit for r in self.completed])
        cols = sum(r.B.shape[1] for r in self.completed)
        if not len(lat):
            return {}
        span = max(r.t_done for r in self.completed) - min(r.t_submit for r in self.completed)
        return {"requests": len(lat), "solves": cols, "solves_per_s": cols / span if span > 0 else None,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3), "launches": self.launches}
