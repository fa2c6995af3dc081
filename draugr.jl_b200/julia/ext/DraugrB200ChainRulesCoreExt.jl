"""
    DraugrB200ChainRulesCoreExt

`ChainRulesCore.rrule` for `DraugrB200.amg_solve_diff`, loaded when
ChainRulesCore is: reverse-mode AD (Zygote and the like) can differentiate
a loss through an AMG solve on the GPU.  The forward pass resets the
hierarchy up with the given nonzeros and solves; the pullback solves the
adjoint system Aᵀλ = x̄ with a transposed cycle on the same hierarchy (P and
Pᵀ swap roles, the coarsest LU is applied transposed) and forms the
per-nonzero gradient -λᵢxⱼ on the device; only the forward solution x is
kept between the passes.  Chain it with the Jacobian of the user's assembly
(cell coefficients -> nonzeros) to get gradients on the cells.
"""
module DraugrB200ChainRulesCoreExt

using DraugrB200
using ChainRulesCore

function ChainRulesCore.rrule(::typeof(DraugrB200.amg_solve_diff), nzval::AbstractVector{Float64},
                              b::AbstractVector{Float64}, h::DraugrB200.AMGHierarchy,
                              config::DraugrB200.AMGConfig=DraugrB200.AMGConfig();
                              tol::Real=1e-12, maxiter::Int=1000, symmetric::Bool=false,
                              precision::Symbol=:fp64)
    x = DraugrB200.amg_solve_diff(nzval, b, h, config; tol=tol, maxiter=maxiter, symmetric=symmetric,
                                  precision=precision)
    function amg_solve_pullback(x̄)
        x̄u = unthunk(x̄)
        x̄u isa AbstractZero && return (NoTangent(), ZeroTangent(), ZeroTangent(), NoTangent(), NoTangent())
        nzval̄, b̄ = DraugrB200.amg_solve_adjoint(collect_like(x̄u, x), x, h, config; tol=tol,
                                                  maxiter=maxiter, symmetric=symmetric, precision=precision)
        return (NoTangent(), nzval̄, b̄, NoTangent(), NoTangent())
    end
    return x, amg_solve_pullback
end

# the cotangent in the same kind of array as x (device memory)
collect_like(x̄::AbstractVector{Float64}, x::AbstractVector{Float64}) = typeof(x̄) === typeof(x) ? x̄ : copyto!(similar(x), x̄)

end # module
