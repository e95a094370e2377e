"""acgpu — the solve phase of Laplacians.jl's approxchol_lap on B200.

Public interface (mirrors the reference's names and keyword semantics):
    approxchol_lap, ApproxCholParams, lap, seed (Random.seed!), approx_chol,
    DeviceLapSolver, components, generators, io (read_graph / writeIJV, LDLinv files).
The solves run in libacgpu.so (CUDA, sm_100a); see include/acgpu.h.
"""
from . import generators, io, tuning
from .solvers import (ApproxCholParams, DeviceLapSolver, GroupSolver, LDLinv, ServeLoop, Ticket, approx_chol,
                      approx_chol_parallel,
                      approxchol_lap, approxchol_lap1,
                      approxchol_lap2, approxchol_sddm,
                      components, lap, null_solver, rng_state, seed, set_rng_state, vec_to_comps)
from .solvers import _init as _solvers_init
from .tuning import autotune

_solvers_init()

__all__ = ["approxchol_lap", "approxchol_lap1", "approxchol_lap2", "approxchol_sddm", "ApproxCholParams", "LDLinv", "DeviceLapSolver", "GroupSolver",
           "ServeLoop", "Ticket",
           "approx_chol", "approx_chol_parallel",
           "lap", "seed", "rng_state", "set_rng_state", "components", "vec_to_comps", "null_solver", "generators",
           "autotune", "tuning", "io"]
