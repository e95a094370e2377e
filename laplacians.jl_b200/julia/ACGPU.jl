# Julia binding of libacgpu.so: the GPU solve phase behind Laplacians.jl's
# approxchol_lap closure.  A maintainer adds this module next to the package
# and swaps the closures built by approxchol_lap1 (src/approxChol.jl:1791-1851)
# for `approxchol_lap1_gpu` below; lapWrapComponents, approxChol and the
# LDLinv type stay as they are, and the factor is built by the reference's own
# elimination for every ApproxCholParams order.
module ACGPU

using Random
using SparseArrays
using Statistics
import Laplacians
import Laplacians: ApproxCholParams, LDLinv, LLmatp, approxChol, lapWrapComponents

const libacgpu = get(ENV, "ACGPU_LIB", joinpath(@__DIR__, "..", "acgpu", "libacgpu.so"))

# acg_solve_info (include/acgpu.h)
struct SolveInfo
    iterations::Int64
    refinements::Int64
    relres::Float64
    best_relres::Float64
    true_relres::Float64
    solve_ms::Float64
    status::Int32
    levels::Int32
end

mutable struct DeviceSolver
    h::Ptr{Cvoid}
    n::Int
end

last_error() = unsafe_string(ccall((:acg_last_error, libacgpu), Cstring, ()))

# acg_create: upload lap(a) and the LDLinv factor (1-based Int64 arrays as Julia stores them).
function DeviceSolver(a::SparseMatrixCSC{Float64,Int64}, ldli::LDLinv{Int64,Float64})
    h = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:acg_create, libacgpu), Cint,
               (Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Float64}, Ptr{Int64}, Ptr{Int64}, Ptr{Int64},
                Ptr{Float64}, Ptr{Float64}, Int64, Cint, Ptr{Cvoid}, Ptr{Ptr{Cvoid}}),
               a.n, a.colptr, a.rowval, a.nzval, ldli.col, ldli.colptr, ldli.rowval, ldli.fval, ldli.d,
               length(ldli.fval), 1, C_NULL, h)
    rc < 0 && error("acg_create: ", last_error())
    s = DeviceSolver(h[], a.n)
    finalizer(s) do s
        ccall((:acg_destroy, libacgpu), Cvoid, (Ptr{Cvoid},), s.h)
    end
    return s
end

# x = f(b): pcg(la, b .- mean(b), LDLsolver; tol, maxits, maxtime, stag_test) on the GPU.
function solve(s::DeviceSolver, b::Vector{Float64}; tol=1e-6, maxits=1000, maxtime=Inf, verbose=false,
               pcgIts=Int[], stag_test=5, precision=0)
    x = similar(b)
    info = Ref{SolveInfo}()
    mi = isfinite(maxits) ? Int64(maxits) : typemax(Int64) >> 1
    rc = ccall((:acg_solve, libacgpu), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Int64, Float64, Int64, Float64, Cint, Cint,
                Ptr{SolveInfo}),
               s.h, b, x, 1, length(b), tol, mi, maxtime, stag_test, precision, info)
    rc < 0 && error("acg_solve: ", last_error())
    if length(pcgIts) > 0
        pcgIts[1] = info[].iterations
    end
    if verbose
        println("PCG stopped after: ", round(info[].solve_ms / 1e3, digits=3), " seconds and ",
                info[].iterations, " iterations with relative error ", info[].relres, ".")
    end
    return x
end

# The factor exactly as the reference's solver for `params` builds it, with the
# reference's own code (and so the same global rand() stream):
#   :deg    approxchol_lapGreedy (src/approxChol.jl:1581-1610), split/merge included
#   :wdeg   approxchol_lapWdeg   (src/approxChol.jl:1676-1733)
#   :random approxchol_lapRandom (src/approxChol.jl:1736-1789)
#   other   approxchol_lapGiven  (src/approxChol.jl:1628-1674)
# as approxchol_lap1 dispatches (src/approxChol.jl:1791-1851).  The fixed-order
# solvers eliminate in a permuted order and relabel the factor back with the
# permutation; the GPU takes that relabelled LDLinv as it is.
function reference_factor(a::SparseMatrixCSC, params::ApproxCholParams)
    if params.order == :deg
        if params.split >= 1 && params.merge < 1
            return approxChol(LLmatp(a, params.split), params.split)
        elseif params.split >= 1 && params.merge >= 1
            return approxChol(LLmatp(a, params.split), params.split, params.merge)
        end
        return approxChol(LLmatp(a))
    end
    if params.order == :wdeg
        v = vec(sum(a, dims=1))
        v = v .* (1 .+ rand(length(v)))
        p = sortperm(v)
    elseif params.order == :random
        p = randperm(size(a, 1))
    else
        return approxChol(Laplacians.LLMatOrd(a))
    end
    ldli = approxChol(Laplacians.LLMatOrd(a, p))
    ip = invperm(p)
    return LDLinv(p[ldli.col], ldli.colptr, p[ldli.rowval], ldli.fval, ldli.d[ip])
end

# Drop-in for approxchol_lap1 (src/approxChol.jl:1791-1851): the same factor as
# the reference's solver for params.order, the same closure signature, the
# solve on the GPU (precision 0: FP64 PCG, the reference algorithm; 1: FP32 PCG
# inside FP64 refinement on the true residual).
function approxchol_lap1_gpu(a::SparseMatrixCSC; tol::Real=1e-6, maxits=1000, maxtime=Inf,
                             verbose=false, pcgIts=Int[], params=ApproxCholParams(), precision=0)
    ldli = reference_factor(a, params)
    s = DeviceSolver(SparseMatrixCSC{Float64,Int64}(a), ldli)
    tol_, maxits_, maxtime_, verbose_, pcgIts_ = tol, maxits, maxtime, verbose, pcgIts
    f(b; tol=tol_, maxits=maxits_, maxtime=maxtime_, verbose=verbose_, pcgIts=pcgIts_) =
        solve(s, b; tol=tol, maxits=maxits, maxtime=maxtime, verbose=verbose, pcgIts=pcgIts,
              stag_test=params.stag_test, precision=precision)
    return f
end

# approxchol_lapGreedy: the :deg factor whatever params.order says, as the reference's.
approxchol_lapGreedy_gpu(a::SparseMatrixCSC; params=ApproxCholParams(), kwargs...) =
    approxchol_lap1_gpu(a; params=ApproxCholParams(:deg, params.stag_test, params.split, params.merge), kwargs...)

# approxchol_lap with the GPU closure, through the reference's component wrapper
# (src/approxChol.jl:1522-1545, src/solverInterface.jl:212-275).
approxchol_lap_gpu(a::SparseMatrixCSC; kwargs...) = lapWrapComponents(approxchol_lap1_gpu, a; kwargs...)

# approxchol_lap2 (src/approxChol.jl:1559-1578): the split/merge factor.
approxchol_lap2_gpu(a::SparseMatrixCSC; params=ApproxCholParams(), kwargs...) =
    approxchol_lap_gpu(a; params=ApproxCholParams(:deg, params.stag_test, 2, 2), kwargs...)

end # module
