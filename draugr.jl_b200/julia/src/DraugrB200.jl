"""
    DraugrB200

Julia front end of libdraugr_b200.so, keeping the names and argument meanings
of Draugr.jl's AMG API (src/setup.jl, src/cycle.jl, src/resetup.jl,
src/types.jl): `amg_setup`, `amg_solve!`, `amg_cycle!`, `amg_resetup!`,
`AMGConfig`, `hypre_default_config`, plus `amg_pcg!` and an `ldiv!`
preconditioner.  Every call is a `ccall` into the C ABI declared in
include/draugr_amg.h and include/draugr_b200.h; setup builds the hierarchy
structure on the CPU inside the library and the solve phase runs on the
current CUDA device.  Vectors may be `Vector{Float64}` (copied to and from
the device by the library) or any array whose `pointer` is a CUDA device
pointer (`CuArray{Float64}` from CUDA.jl), which is passed straight through.
"""
module DraugrB200

using LinearAlgebra
using SparseArrays

export AMGConfig, hypre_default_config, AMGHierarchy
export amg_setup, amg_solve!, amg_cycle!, amg_resetup!, amg_pcg!
export amg_bicgstab!, amg_fgmres!, amg_refine!, amg_pcg_block!, nz_gradient!
export amg_solve_diff, amg_solve_adjoint, amg_resetup_values!
export amg_batch_setup, amg_pcg_batched!
export DraugrB200Preconditioner

const libdraugr = get(ENV, "DRAUGR_B200_LIB", joinpath(@__DIR__, "..", "..", "libdraugr_b200.so"))

struct DraugrError <: Exception
    msg::String
end
Base.showerror(io::IO, e::DraugrError) = print(io, "DraugrB200: ", e.msg)

last_error() = unsafe_string(ccall((:draugr_amg_last_error, libdraugr), Cstring, ()))
check(rc::Integer, what) = rc < 0 ? throw(DraugrError(string(what, ": ", last_error()))) : rc

# ---------------------------------------------------------------- configuration
# Type tags mirror src/types.jl; they are turned into the JSON accepted by
# draugr_amg_config_from_json (same keys as src/cfunction_interface.jl).
abstract type InterpolationType end
struct DirectInterpolation <: InterpolationType
    trunc_factor::Float64
end
DirectInterpolation() = DirectInterpolation(0.0)
struct StandardInterpolation <: InterpolationType
    trunc_factor::Float64
end
StandardInterpolation() = StandardInterpolation(0.0)
struct ExtendedIInterpolation <: InterpolationType
    trunc_factor::Float64
    max_elements::Int
    norm_p::Int
    rescale::Bool
end
ExtendedIInterpolation() = ExtendedIInterpolation(0.0, 0, 1, false)
ExtendedIInterpolation(tf::Real) = ExtendedIInterpolation(Float64(tf), 0, 1, false)

abstract type CoarseningAlgorithm end
struct AggregationCoarsening <: CoarseningAlgorithm
    θ::Float64
    filtering::Bool
    filter_tol::Float64
end
AggregationCoarsening(θ::Real=0.25) = AggregationCoarsening(θ, false, 0.1)
struct PMISCoarsening <: CoarseningAlgorithm
    θ::Float64
    interpolation::InterpolationType
end
PMISCoarsening(θ::Real=0.25) = PMISCoarsening(θ, DirectInterpolation())
struct HMISCoarsening <: CoarseningAlgorithm
    θ::Float64
    interpolation::InterpolationType
end
struct RSCoarsening <: CoarseningAlgorithm
    θ::Float64
    interpolation::InterpolationType
end
RSCoarsening(θ::Real=0.25) = RSCoarsening(θ, DirectInterpolation())
HMISCoarsening(θ::Real=0.25) = HMISCoarsening(θ, DirectInterpolation())
struct AggressiveCoarsening <: CoarseningAlgorithm
    θ::Float64
    base::Symbol
    interpolation::InterpolationType
end
AggressiveCoarsening(θ::Real=0.25, base::Symbol=:pmis) = AggressiveCoarsening(θ, base, ExtendedIInterpolation())
struct SmoothedAggregationCoarsening <: CoarseningAlgorithm
    θ::Float64
    ω::Float64
end
SmoothedAggregationCoarsening(θ::Real=0.25) = SmoothedAggregationCoarsening(θ, 2 / 3)

abstract type SmootherType end
for (T, name) in ((:JacobiSmootherType, "jacobi"), (:L1JacobiSmootherType, "l1_jacobi"),
                  (:ColoredGaussSeidelType, "colored_gs"), (:L1ColoredGaussSeidelType, "l1_colored_gs"),
                  (:SerialGaussSeidelType, "serial_gs"), (:L1SerialGaussSeidelType, "l1_serial_gs"),
                  (:SPAI0SmootherType, "spai0"), (:SPAI1SmootherType, "spai1"),
                  (:ChebyshevSmootherType, "chebyshev"), (:ILU0SmootherType, "ilu0"),
                  (:SerialILU0SmootherType, "serial_ilu0"))
    @eval begin
        struct $T <: SmootherType end
        smoother_name(::$T) = $name
        export $T
    end
end
export AggregationCoarsening, PMISCoarsening, HMISCoarsening, RSCoarsening, AggressiveCoarsening,
       SmoothedAggregationCoarsening, DirectInterpolation, StandardInterpolation,
       ExtendedIInterpolation

jstr(x::AbstractString) = "\"" * replace(x, "\"" => "\\\"") * "\""
jstr(x::Bool) = x ? "true" : "false"
jstr(x::Real) = string(x)

interp_json(i::DirectInterpolation) = "{\"type\":\"direct\",\"trunc_factor\":$(i.trunc_factor)}"
interp_json(i::StandardInterpolation) = "{\"type\":\"standard\",\"trunc_factor\":$(i.trunc_factor)}"
interp_json(i::ExtendedIInterpolation) =
    "{\"type\":\"extended_i\",\"trunc_factor\":$(i.trunc_factor),\"max_elements\":$(i.max_elements)," *
    "\"norm_p\":$(i.norm_p),\"rescale\":$(jstr(i.rescale))}"

coarsening_json(c::AggregationCoarsening) = ("aggregation", c.θ, nothing,
    ",\"aggregation_filtering\":$(jstr(c.filtering)),\"filter_tol\":$(c.filter_tol)")
coarsening_json(c::SmoothedAggregationCoarsening) = ("smoothed_aggregation", c.θ, nothing, ",\"sa_omega\":$(c.ω)")
coarsening_json(c::PMISCoarsening) = ("pmis", c.θ, c.interpolation, "")
coarsening_json(c::HMISCoarsening) = ("hmis", c.θ, c.interpolation, "")
coarsening_json(c::RSCoarsening) = ("rs", c.θ, c.interpolation, "")
coarsening_json(c::AggressiveCoarsening) = ("aggressive_" * String(c.base), c.θ, c.interpolation, "")

"""
    AMGConfig(; kwargs...)

Same keywords and defaults as Draugr.jl's `AMGConfig` (src/types.jl:514-536),
plus `seed` for the random PMIS/HMIS measures.
"""
struct AMGConfig
    json::String
    handle::Int32
    pre_smoothing_steps::Int
    post_smoothing_steps::Int
end

function AMGConfig(; coarsening::CoarseningAlgorithm=HMISCoarsening(0.5, ExtendedIInterpolation()),
                   smoother::SmootherType=L1ColoredGaussSeidelType(), max_levels::Int=20,
                   max_coarse_size::Int=50, pre_smoothing_steps::Int=1, post_smoothing_steps::Int=1,
                   jacobi_omega::Float64=2.0 / 3.0, verbose::Union{Bool,Int}=0,
                   initial_coarsening::CoarseningAlgorithm=coarsening,
                   initial_coarsening_levels::Int=0, max_row_sum::Float64=1.0,
                   cycle_type::Symbol=:V, coarse_solve_on_cpu::Bool=false,
                   seed::Union{Nothing,Integer}=nothing)
    @assert cycle_type in (:V, :W) "cycle_type must be :V or :W"
    name, θ, ip, extra = coarsening_json(coarsening)
    iname, iθ, iip, _ = coarsening_json(initial_coarsening)
    js = "{\"coarsening\":$(jstr(name)),\"theta\":$(θ)" *
         (ip === nothing ? "" : ",\"interpolation\":" * interp_json(ip)) * extra *
         ",\"initial_coarsening\":$(jstr(iname)),\"initial_theta\":$(iθ)" *
         (iip === nothing ? "" : ",\"initial_interpolation\":" * interp_json(iip)) *
         ",\"smoother\":{\"type\":$(jstr(smoother_name(smoother))),\"omega\":$(jacobi_omega)}" *
         ",\"max_levels\":$(max_levels),\"max_coarse_size\":$(max_coarse_size)" *
         ",\"pre_smoothing_steps\":$(pre_smoothing_steps),\"post_smoothing_steps\":$(post_smoothing_steps)" *
         ",\"verbose\":$(Int(verbose)),\"initial_coarsening_levels\":$(initial_coarsening_levels)" *
         ",\"max_row_sum\":$(max_row_sum),\"cycle\":$(jstr(lowercase(String(cycle_type))))" *
         ",\"coarse_solve_on_cpu\":$(jstr(coarse_solve_on_cpu))" *
         (seed === nothing ? "" : ",\"seed\":$(seed)") * "}"
    h = check(ccall((:draugr_amg_config_from_json, libdraugr), Int32, (Cstring,), js),
              "draugr_amg_config_from_json")
    return AMGConfig(js, h, pre_smoothing_steps, post_smoothing_steps)
end

"""hypre_default_config (src/types.jl:569-584)."""
function hypre_default_config(; θ::Float64=0.5, agg_num_levels::Int=1,
                              agg_trunc_factor::Float64=0.3, kwargs...)
    interp = ExtendedIInterpolation(agg_trunc_factor)
    return AMGConfig(; coarsening=HMISCoarsening(θ, interp),
                     initial_coarsening=AggressiveCoarsening(θ, :hmis, interp),
                     initial_coarsening_levels=agg_num_levels, kwargs...)
end

# ---------------------------------------------------------------- hierarchy
mutable struct AMGHierarchy
    handle::Int32
    n::Int
    function AMGHierarchy(h::Int32, n::Int)
        H = new(h, n)
        finalizer(H) do H
            H.handle > 0 && ccall((:draugr_amg_free, libdraugr), Int32, (Int32,), H.handle)
            H.handle = -1
        end
        return H
    end
end

# CSR arrays (1-based Int32) of a SparseMatrixCSC, as csr_from_csc does.
function csr_arrays(A::SparseMatrixCSC)
    At = sparse(transpose(A))
    return Int32.(At.colptr), Int32.(At.rowval), Vector{Float64}(At.nzval)
end

"""
    amg_setup(A, config=AMGConfig(); allow_partial_resetup=true) -> AMGHierarchy
"""
function amg_setup(A::SparseMatrixCSC, config::AMGConfig=AMGConfig();
                   allow_partial_resetup::Bool=true)
    n = size(A, 1)
    rp, cv, nz = csr_arrays(A)
    h = check(ccall((:draugr_amg_setup, libdraugr), Int32,
                    (Int32, Int32, Ptr{Int32}, Ptr{Int32}, Ptr{Float64}, Int32, Int32, Int32),
                    n, length(nz), rp, cv, nz, config.handle, 1, allow_partial_resetup),
              "amg_setup")
    return AMGHierarchy(h, n)
end

"""
    amg_resetup!(h, A, config; partial=true, allow_partial_resetup=true) -> h
"""
function amg_resetup!(h::AMGHierarchy, A::SparseMatrixCSC, config::AMGConfig=AMGConfig();
                      partial::Bool=true, allow_partial_resetup::Bool=true)
    rp, cv, nz = csr_arrays(A)
    check(ccall((:draugr_amg_resetup, libdraugr), Int32,
                (Int32, Int32, Int32, Ptr{Int32}, Ptr{Int32}, Ptr{Float64}, Int32, Int32, Int32, Int32),
                h.handle, size(A, 1), length(nz), rp, cv, nz, config.handle, 1, partial,
                allow_partial_resetup), "amg_resetup!")
    return h
end

# Host vectors go through the host-pointer entry points; anything else is
# taken to be device memory (e.g. CuArray) and its pointer passed as is.
isdevice(x) = !(x isa Array)
rawptr(x) = reinterpret(Ptr{Float64}, UInt(pointer(x)))

"""
    amg_cycle!(x, b, h, config) -> x
"""
function amg_cycle!(x::AbstractVector{Float64}, b::AbstractVector{Float64}, h::AMGHierarchy,
                    config::AMGConfig=AMGConfig())
    if isdevice(x)
        check(ccall((:draugr_b200_cycle_device, libdraugr), Int32,
                    (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32),
                    h.handle, length(x), rawptr(x), rawptr(b), config.handle), "amg_cycle!")
    else
        check(ccall((:draugr_amg_cycle, libdraugr), Int32,
                    (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32),
                    h.handle, length(x), x, b, config.handle), "amg_cycle!")
    end
    return x
end

"""
    amg_solve!(x, b, h, config; tol=1e-10, maxiter=100) -> (x, niter)
"""
function amg_solve!(x::AbstractVector{Float64}, b::AbstractVector{Float64}, h::AMGHierarchy,
                    config::AMGConfig=AMGConfig(); tol::Real=1e-10, maxiter::Int=100)
    it = if isdevice(x)
        ccall((:draugr_b200_solve_device, libdraugr), Int32,
              (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32),
              h.handle, length(x), rawptr(x), rawptr(b), config.handle, tol, maxiter)
    else
        ccall((:draugr_amg_solve, libdraugr), Int32,
              (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32),
              h.handle, length(x), x, b, config.handle, tol, maxiter)
    end
    return x, Int(check(it, "amg_solve!"))
end

"""
    amg_pcg!(x, b, h, config; tol=1e-8, maxiter=500, precision=:fp64) -> (x, niter, relres)

Conjugate gradients preconditioned by one AMG cycle per iteration;
`precision=:mixed` runs the cycle on FP32 copies of the hierarchy with the
outer iteration in FP64.
"""
function amg_pcg!(x::AbstractVector{Float64}, b::AbstractVector{Float64}, h::AMGHierarchy,
                  config::AMGConfig=AMGConfig(); tol::Real=1e-8, maxiter::Int=500,
                  precision::Symbol=:fp64)
    prec = precision === :mixed ? Int32(1) : Int32(0)
    rel = Ref{Float64}(0.0)
    it = GC.@preserve x b if isdevice(x)
        ccall((:draugr_b200_pcg_device, libdraugr), Int32,
              (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32, Int32, Ref{Float64}),
              h.handle, length(x), rawptr(x), rawptr(b), config.handle, tol, maxiter, prec, rel)
    else
        ccall((:draugr_b200_pcg, libdraugr), Int32,
              (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32, Int32, Ref{Float64}),
              h.handle, length(x), pointer(x), pointer(b), config.handle, tol, maxiter, prec, rel)
    end
    return x, Int(check(it, "amg_pcg!")), rel[]
end

"""
    amg_bicgstab!(x, b, h, config; tol=1e-8, maxiter=500, transpose=false, precision=:fp64) -> (x, niter, relres)

BiCGStab preconditioned (on the right) by one cycle, for nonsymmetric
systems; `transpose=true` solves Aᵀx = b on the transposed hierarchy (the
adjoint solve of a gradient).  Every level must use Jacobi, l1-Jacobi or
SPAI(0) smoothing for the transposed cycle.  `precision=:mixed` runs the
cycle on FP32 copies (of the hierarchy or its transpose) with the BiCGStab
vectors, products and dots in FP64.
"""
function amg_bicgstab!(x::AbstractVector{Float64}, b::AbstractVector{Float64}, h::AMGHierarchy,
                       config::AMGConfig=AMGConfig(); tol::Real=1e-8, maxiter::Int=500,
                       transpose::Bool=false, precision::Symbol=:fp64)
    rel = Ref{Float64}(0.0)
    tr = Int32(transpose)
    prec = precision === :mixed ? Int32(1) : Int32(0)
    it = GC.@preserve x b if isdevice(x)
        ccall((:draugr_b200_bicgstab_device, libdraugr), Int32,
              (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32, Int32, Int32, Ref{Float64}),
              h.handle, length(x), rawptr(x), rawptr(b), config.handle, tol, maxiter, tr, prec, rel)
    else
        ccall((:draugr_b200_bicgstab, libdraugr), Int32,
              (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32, Int32, Int32, Ref{Float64}),
              h.handle, length(x), pointer(x), pointer(b), config.handle, tol, maxiter, tr, prec, rel)
    end
    return x, Int(check(it, "amg_bicgstab!")), rel[]
end

"""
    amg_fgmres!(x, b, h, config; tol=1e-8, maxiter=500, restart=30, precision=:fp64) -> (x, niter, relres)

Flexible GMRES(restart), right-preconditioned by one cycle per iteration
(FP64, or the FP32 cycle with `precision=:mixed`), FP64 Arnoldi.  For
symmetric and nonsymmetric systems.
"""
function amg_fgmres!(x::AbstractVector{Float64}, b::AbstractVector{Float64}, h::AMGHierarchy,
                     config::AMGConfig=AMGConfig(); tol::Real=1e-8, maxiter::Int=500, restart::Int=30,
                     precision::Symbol=:fp64)
    rel = Ref{Float64}(0.0)
    prec = precision === :mixed ? Int32(1) : Int32(0)
    it = GC.@preserve x b if isdevice(x)
        ccall((:draugr_b200_fgmres_device, libdraugr), Int32,
              (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32, Int32, Int32, Ref{Float64}),
              h.handle, length(x), rawptr(x), rawptr(b), config.handle, tol, maxiter, restart, prec, rel)
    else
        ccall((:draugr_b200_fgmres, libdraugr), Int32,
              (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32, Int32, Int32, Ref{Float64}),
              h.handle, length(x), pointer(x), pointer(b), config.handle, tol, maxiter, restart, prec, rel)
    end
    return x, Int(check(it, "amg_fgmres!")), rel[]
end

"""
    amg_refine!(x, b, h, config; tol=1e-8, max_outer=20, inner_tol=1e-4, inner_maxiter=500,
                inner=:pcg, precision=:mixed) -> (x, steps, inner_iterations, relres)

Iterative refinement: FP64 residual r = b - A x, the correction A d = r
solved to `inner_tol` by AMG-PCG (`inner=:pcg`) or FGMRES (`inner=:fgmres`)
with the FP32 (`:mixed`) or FP64 cycle, x += d, until the FP64 relative
residual is below `tol`.
"""
function amg_refine!(x::AbstractVector{Float64}, b::AbstractVector{Float64}, h::AMGHierarchy,
                     config::AMGConfig=AMGConfig(); tol::Real=1e-8, max_outer::Int=20,
                     inner_tol::Real=1e-4, inner_maxiter::Int=500, inner::Symbol=:pcg,
                     precision::Symbol=:mixed)
    rel = Ref{Float64}(0.0)
    its = Ref{Int32}(0)
    prec = precision === :mixed ? Int32(1) : Int32(0)
    meth = inner === :fgmres ? Int32(1) : Int32(0)
    st = GC.@preserve x b if isdevice(x)
        ccall((:draugr_b200_refine_device, libdraugr), Int32,
              (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32, Float64, Int32, Int32, Int32,
               Ref{Float64}, Ref{Int32}),
              h.handle, length(x), rawptr(x), rawptr(b), config.handle, tol, max_outer, inner_tol,
              inner_maxiter, meth, prec, rel, its)
    else
        ccall((:draugr_b200_refine, libdraugr), Int32,
              (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32, Float64, Int32, Int32, Int32,
               Ref{Float64}, Ref{Int32}),
              h.handle, length(x), pointer(x), pointer(b), config.handle, tol, max_outer, inner_tol,
              inner_maxiter, meth, prec, rel, its)
    end
    return x, Int(check(st, "amg_refine!")), Int(its[]), rel[]
end

"""
    amg_pcg_block!(X, B, h, config; tol=1e-8, maxiter=500, precision=:mixed) -> (X, iters, relres)

CG for k ≤ 32 right-hand sides of one matrix at once, each product with a
level matrix serving all k.  `X` and `B` are device matrices of size
(k, n): column i holds row i's k entries (the library's n × k row-major
layout).  Returns per-column iteration counts and relative residuals.
"""
function amg_pcg_block!(X::AbstractMatrix{Float64}, B::AbstractMatrix{Float64}, h::AMGHierarchy,
                        config::AMGConfig=AMGConfig(); tol::Real=1e-8, maxiter::Int=500,
                        precision::Symbol=:mixed)
    k, n = size(X)
    size(B) == (k, n) || throw(DimensionMismatch("X and B must have the same size"))
    its = zeros(Int32, k)
    rel = zeros(Float64, k)
    prec = precision === :mixed ? Int32(1) : Int32(0)
    rc = GC.@preserve X B ccall((:draugr_b200_pcg_block_device, libdraugr), Int32,
                                (Int32, Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32,
                                 Int32, Ptr{Int32}, Ptr{Float64}),
                                h.handle, n, k, rawptr(X), rawptr(B), config.handle, tol, maxiter, prec,
                                its, rel)
    check(rc, "amg_pcg_block!")
    return X, Int.(its), rel
end

"""
    nz_gradient!(grad, h, x, λ) -> grad

dL/da_ij = -λ_i x_j for the finest matrix's nonzeros, in CSR order (device
vectors; grad has nnz entries), with x = A⁻¹b and λ = A⁻ᵀ dL/dx.
"""
function nz_gradient!(grad::AbstractVector{Float64}, h::AMGHierarchy, x::AbstractVector{Float64},
                      λ::AbstractVector{Float64})
    rc = GC.@preserve grad x λ ccall((:draugr_b200_nz_gradient_device, libdraugr), Int32,
                                     (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                                     h.handle, length(x), rawptr(x), rawptr(λ), rawptr(grad))
    check(rc, "nz_gradient!")
    return grad
end

"""
    amg_resetup_values!(h, nzval) -> h

Partial resetup from new values of the finest matrix in CSR order (the
setup's pattern), on the device (`nzval` a device array) or copied there.
"""
function amg_resetup_values!(h::AMGHierarchy, nzval::AbstractVector{Float64})
    GC.@preserve nzval begin
        if isdevice(nzval)
            check(ccall((:draugr_b200_resetup_values_device, libdraugr), Int32, (Int32, Int64, Ptr{Float64}),
                        h.handle, length(nzval), rawptr(nzval)), "amg_resetup_values!")
        else
            throw(ArgumentError("amg_resetup_values! takes device values; use amg_resetup! for a host matrix"))
        end
    end
    return h
end

"""
    amg_solve_diff(nzval, b, h, config; tol=1e-12, maxiter=1000, symmetric=false, precision=:fp64) -> x

x = A(nzval)⁻¹ b, where nzval are the finest matrix's nonzeros in CSR order
(the setup pattern): a partial resetup with `nzval`, then AMG-PCG
(`symmetric`) or AMG-BiCGStab.  Differentiable: the package extension for
ChainRulesCore defines its `rrule`, whose pullback solves Aᵀλ = x̄ on the
transposed hierarchy and returns (nzval̄ = -λᵢxⱼ per nonzero, b̄ = λ).
`nzval`, `b` and the result are device arrays (e.g. CuArray{Float64}).
"""
function amg_solve_diff(nzval::AbstractVector{Float64}, b::AbstractVector{Float64}, h::AMGHierarchy,
                        config::AMGConfig=AMGConfig(); tol::Real=1e-12, maxiter::Int=1000,
                        symmetric::Bool=false, precision::Symbol=:fp64)
    amg_resetup_values!(h, nzval)
    x = similar(b)
    fill!(x, 0.0)
    if symmetric
        amg_pcg!(x, b, h, config; tol=tol, maxiter=maxiter, precision=precision)
    else
        amg_bicgstab!(x, b, h, config; tol=tol, maxiter=maxiter, precision=precision)
    end
    return x
end

"""
    amg_solve_adjoint(x̄, x, h, config; tol, maxiter, symmetric, precision) -> (nzval̄, b̄)

The pullback of `amg_solve_diff` at its result x: λ = A⁻ᵀ x̄ (PCG when
symmetric, else BiCGStab on the transposed hierarchy), b̄ = λ and
nzval̄ᵢⱼ = -λᵢ xⱼ over the nonzeros (draugr_b200_nz_gradient_device).  Only
x is needed from the forward pass.
"""
function amg_solve_adjoint(x̄::AbstractVector{Float64}, x::AbstractVector{Float64}, h::AMGHierarchy,
                           config::AMGConfig=AMGConfig(); tol::Real=1e-12, maxiter::Int=1000,
                           symmetric::Bool=false, precision::Symbol=:fp64)
    λ = similar(x)
    fill!(λ, 0.0)
    if symmetric
        amg_pcg!(λ, x̄, h, config; tol=tol, maxiter=maxiter, precision=precision)
    else
        amg_bicgstab!(λ, x̄, h, config; tol=tol, maxiter=maxiter, transpose=true, precision=precision)
    end
    info = zeros(Int64, 10)
    check(ccall((:draugr_b200_level_info, libdraugr), Int32, (Int32, Int32, Ptr{Int64}), h.handle, 0, info),
          "amg_solve_adjoint")
    grad = similar(x, Int(info[2]))
    nz_gradient!(grad, h, x, λ)
    return grad, λ
end

"""
    amg_batch_setup(hs::Vector{AMGHierarchy}) -> (batch::AMGHierarchy, offsets::Vector{Int})

Merge independent systems' hierarchies level by level into one batch on the
current device; system s occupies rows offsets[s]+1 : offsets[s+1] of the
batch's vectors.  The systems' own hierarchies stay usable.
"""
function amg_batch_setup(hs::Vector{AMGHierarchy})
    handles = Int32[h.handle for h in hs]
    b = check(ccall((:draugr_b200_batch_setup, libdraugr), Int32, (Int32, Ptr{Int32}),
                    length(handles), handles), "amg_batch_setup")
    offs = zeros(Int64, length(hs) + 1)
    check(ccall((:draugr_b200_batch_offsets, libdraugr), Int32, (Int32, Ptr{Int64}), b, offs),
          "amg_batch_setup")
    return AMGHierarchy(b, Int(offs[end])), Int.(offs)
end

"""
    amg_pcg_batched!(x, b, batch, config; tol=1e-8, maxiter=500, precision=:mixed) -> (x, iters, relres)

AMG-PCG on every system of a batch at once (device vectors holding all
systems' rows): one launch per cycle stage for all systems, per-system step
sizes and convergence.  Returns per-system iterations and relative
residuals.
"""
function amg_pcg_batched!(x::AbstractVector{Float64}, b::AbstractVector{Float64}, batch::AMGHierarchy,
                          config::AMGConfig=AMGConfig(); tol::Real=1e-8, maxiter::Int=500,
                          precision::Symbol=:mixed)
    ns = check(ccall((:draugr_b200_batch_offsets, libdraugr), Int32, (Int32, Ptr{Int64}), batch.handle,
                     C_NULL), "amg_pcg_batched!")
    its = zeros(Int32, ns)
    rel = zeros(Float64, ns)
    prec = precision === :mixed ? Int32(1) : Int32(0)
    rc = GC.@preserve x b ccall((:draugr_b200_batch_pcg_device, libdraugr), Int32,
                                (Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Float64, Int32, Int32,
                                 Ptr{Int32}, Ptr{Float64}),
                                batch.handle, length(x), rawptr(x), rawptr(b), config.handle, tol, maxiter,
                                prec, its, rel)
    check(rc, "amg_pcg_batched!")
    return x, Int.(its), rel
end

"""
    DraugrB200Preconditioner(h, config)

`ldiv!(x, P, b)` zeroes x and applies one cycle, like Draugr.jl's
`preconditioner_apply!` (src/preconditioner.jl:76-80), for Krylov.jl or
LinearSolve.jl.
"""
struct DraugrB200Preconditioner
    h::AMGHierarchy
    config::AMGConfig
end

function LinearAlgebra.ldiv!(x::AbstractVector{Float64}, P::DraugrB200Preconditioner,
                             b::AbstractVector{Float64})
    fill!(x, 0.0)
    return amg_cycle!(x, b, P.h, P.config)
end

end # module
