"""
    MSLRB200ChainRules

`ChainRulesCore.rrule` for the unrolled-POGM loss of MSLRB200, so that Zygote
(or any ChainRules-aware AD) can differentiate a loss of the per-scale
log-weights log λ_k through `run_recon`'s iteration.  Load after MSLRB200 in
an environment that has ChainRulesCore:

    include("MSLRB200.jl"); include("MSLRB200ChainRules.jl")
    using .MSLRB200, .MSLRB200ChainRules
    ℓ = unrolled_loss(ctx, logλ, X_true, 10, 2.0)     # differentiable in logλ
"""
module MSLRB200ChainRules

using ChainRulesCore
using CUDA
using ..MSLRB200

export unrolled_loss

"""½‖Σ_k X_niter[..,k] − X_true‖² after `niter` POGM iterations with λ = exp.(logλ)."""
function unrolled_loss(ctx::MSLRContext, logλ::AbstractVector{<:Real}, X_true::CuArray{ComplexF32},
                       niter::Integer, L::Real)
    set_lambdas!(ctx, exp.(logλ))
    return first(pogm_grad(ctx, X_true, niter, L))
end

function ChainRulesCore.rrule(::typeof(unrolled_loss), ctx::MSLRContext,
                              logλ::AbstractVector{<:Real}, X_true::CuArray{ComplexF32},
                              niter::Integer, L::Real)
    set_lambdas!(ctx, exp.(logλ))
    loss, grad, X, _ = pogm_grad(ctx, X_true, niter, L)
    # ∂loss/∂X_true = −(Σ_k X_k − X_true): X does not depend on X_true
    pullback(ȳ) = (NoTangent(), NoTangent(), ȳ .* grad,
                   @thunk(-ȳ .* (dropdims(sum(X; dims=5); dims=5) .- X_true)),
                   NoTangent(), NoTangent())
    return loss, pullback
end

end # module
