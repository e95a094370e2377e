# Julia binding of libacgpu.so: the GPU solve phase behind Laplacians.jl's
# approxchol_lap closure.  A maintainer adds this module next to the package
# and swaps the closure built by approxchol_lapGreedy (src/approxChol.jl:1581-1626)
# for `approxchol_lapGreedy_gpu` below; lapWrapComponents, approxChol and the
# LDLinv type stay as they are.
module ACGPU

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

# Drop-in for approxchol_lapGreedy: same factor (host elimination, same global
# rand() stream), same closure signature, the solve on the GPU.
function approxchol_lapGreedy_gpu(a::SparseMatrixCSC; tol::Real=1e-6, maxits=1000, maxtime=Inf,
                                  verbose=false, pcgIts=Int[], params=ApproxCholParams())
    llmat = LLmatp(a)
    ldli = approxChol(llmat)
    s = DeviceSolver(SparseMatrixCSC{Float64,Int64}(a), ldli)
    tol_, maxits_, maxtime_, verbose_, pcgIts_ = tol, maxits, maxtime, verbose, pcgIts
    f(b; tol=tol_, maxits=maxits_, maxtime=maxtime_, verbose=verbose_, pcgIts=pcgIts_) =
        solve(s, b; tol=tol, maxits=maxits, maxtime=maxtime, verbose=verbose, pcgIts=pcgIts,
              stag_test=params.stag_test)
    return f
end

# approxchol_lap with the GPU closure, through the reference's component wrapper.
approxchol_lap_gpu(a::SparseMatrixCSC; kwargs...) = lapWrapComponents(approxchol_lapGreedy_gpu, a; kwargs...)

end # module
