"""Autotuner for the solver's tuning knobs (`acg_options`, include/acgpu.h).

The knobs change how `acg_create` lays out the work, not what is computed:
the heavy-task thresholds of the sweeps' task tables, the size of the dense
tail, the resident sweep blocks per SM and the sweep vectors' layout.  Their
best values depend on the graph (its LDLinv DAG: depth, width profile, row
lengths) and on the batch width, so the tuner measures them on the graph at
hand: it builds a solver per candidate, times one PCG iteration's kernels with
`acg_time_kernels` / `acg_time_kernels_batch` (CUDA events on the device) and
walks the knobs one at a time from the defaults (coordinate descent), keeping
a change only when it is faster by more than `min_gain`.

The reference has no counterpart: its solve has no layout to tune.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

__all__ = ["TuneResult", "default_space", "coordinate_descent", "autotune", "iteration_ms"]


@dataclass
class TuneResult:
    options: dict                      # the chosen knobs (only those that differ from the defaults)
    ms: float                          # their measured time per iteration
    baseline_ms: float                 # the defaults' time per iteration
    trials: list = field(default_factory=list)  # (options, ms) for every candidate measured

    @property
    def speedup(self) -> float:
        return self.baseline_ms / self.ms if self.ms > 0 else 1.0


def default_space(nrhs: int) -> dict:
    """Candidate values per knob, defaults first (0 = the library's automatic choice)."""
    if nrhs > 1:
        return {
            "dense_tail": [0, 1024, 2048, 8192, -1],
            "batch_fwd_heavy": [0, 4, 16, 32],
            "batch_bwd_heavy": [0, 4, 16, 32],
            "batch_blocks_per_sm": [0, 1],
        }
    return {
        "dense_tail": [0, 1024, 2048, 8192, -1],
        "sweep_heavy": [0, 8, 32, 64],
        "sweep_blocks_per_sm": [0, 2],
    }


def coordinate_descent(measure: Callable[[dict], float], space: dict, rounds: int = 2,
                       min_gain: float = 0.02) -> TuneResult:
    """Minimise measure(options) one knob at a time.  `space` maps each knob to
    its candidate values, the first being the default.  A value replaces the
    current one only when it is faster by more than `min_gain` (relative)."""
    cache: dict = {}
    trials = []

    def timed(opts: dict) -> float:
        key = tuple(sorted(opts.items()))
        if key not in cache:
            cache[key] = float(measure(dict(opts)))
            trials.append((dict(opts), cache[key]))
        return cache[key]

    current = {k: v[0] for k, v in space.items()}
    base = timed(current)
    best = base
    for _ in range(rounds):
        changed = False
        for knob, values in space.items():
            for v in values:
                if v == current[knob]:
                    continue
                cand = dict(current, **{knob: v})
                t = timed(cand)
                if t < best * (1.0 - min_gain):
                    best, current, changed = t, cand, True
        if not changed:
            break
    chosen = {k: v for k, v in current.items() if v != space[k][0]}
    return TuneResult(options=chosen, ms=best, baseline_ms=base, trials=trials)


def iteration_ms(dev, nrhs: int, precision: str, reps: int = 3) -> float:
    """Device time of one PCG iteration's dominant kernels: the mat-vec and both
    preconditioner sweeps (dense tail included) for `nrhs` columns."""
    if nrhs > 1:
        kt = dev.time_kernels_batch(nrhs, precision, reps=reps)
    else:
        kt = dev.time_kernels(precision, reps=reps)
    return kt["spmv_ms"] + kt["forward_ms"] + kt["backward_ms"]


def autotune(a, ldli, nrhs: int = 1, precision: str = "mixed", space: dict | None = None, rounds: int = 2,
             min_gain: float = 0.02, reps: int = 3, build: Callable | None = None) -> TuneResult:
    """Tune the solver's knobs for graph `a` with factor `ldli`, `nrhs`
    right-hand sides per solve and `precision` ("mixed" or "fp64").  Returns
    the option dict to pass as `DeviceLapSolver(a, ldli, options=...)`.
    `build(options)` may replace the solver constructor (it must return an
    object with time_kernels / time_kernels_batch and close)."""
    from .solvers import DeviceLapSolver

    if build is None:
        def build(opts):
            return DeviceLapSolver(a, ldli, options={k: v for k, v in opts.items() if v != 0})

    def measure(opts: dict) -> float:
        dev = build(opts)
        try:
            return iteration_ms(dev, nrhs, precision, reps)
        finally:
            dev.close()

    return coordinate_descent(measure, space or default_space(nrhs), rounds=rounds, min_gain=min_gain)
