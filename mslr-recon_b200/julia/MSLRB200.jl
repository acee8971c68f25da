"""
    MSLRB200

Julia binding of `libmslr.so` (the C ABI in `include/mslr.h`): drop-in
replacements for the per-iteration path of `run_recon`
(`scripts/reconstruct.jl`) — the SENSE operator `Asense_gpu`
(`src/sense_gpu.jl:56-108`), `dc_cost_grad` (`scripts/reconstruct.jl:180-183`),
`patchSVST_gpu` (`src/sense_gpu.jl:138-160`), `pogm_mod` with `mom=:pogm,
restart=:gr` (`src/mirt_mod.jl:74-188`) and `poweriter_mod`
(`src/mirt_mod.jl:215-238`).

Arrays are `CuArray{ComplexF32}` in the reference's column-major layouts:
image `(Nx,Ny,Nz,Nt)`, `X` `(Nx,Ny,Nz,Nt,Ns)`, coil maps `(Nx,Ny,Nz,Nc)`,
k-space `(K,Nc,Nt)`, sample indices `(K,Nt)` 1-based `Int32`.  Every call
runs on CUDA.jl's task-local stream.  Library errors are raised as
`ArgumentError` (bad arguments, as the reference does) or `MSLRError`.
"""
module MSLRB200

using CUDA

export MSLRContext, pogm_mod!, sense_forward!, sense_adjoint!, dc_cost_grad!, patch_svst!,
       pogm_run!, cost, sync!, power_iter, mslr_lambdas, set_lambdas!, pogm_grad, mslr_sampling

const libmslr = get(ENV, "MSLR_LIB", joinpath(@__DIR__, "..", "libmslr.so"))

struct MSLRError <: Exception
    code::Int32
    msg::String
end

const FORM_PLAIN = Int32(0)
const FORM_TUNED = Int32(1)
const FORM_TF32 = Int32(2)

_stream() = CUDA.stream().handle   # cudaStream_t of the task-local stream

function _check(rc::Integer, h::Ptr{Cvoid}=C_NULL)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:mslr_last_error, libmslr), Cstring, (Ptr{Cvoid},), h))
    rc == 1 && throw(ArgumentError(msg))
    throw(MSLRError(Int32(rc), msg))
end

"""
    MSLRContext(N, Nc, Nt, K, patch_sizes, strides; form=:tuned)

The state `run_recon` builds (scripts/reconstruct.jl:133-214) for
`length(patch_sizes)` scales.  Free with `close(ctx)` (or let the GC do it).
"""
mutable struct MSLRContext
    h::Ptr{Cvoid}
    N::NTuple{3,Int}
    Nc::Int
    Nt::Int
    K::Int
    Ns::Int
    niter::Int
end

function MSLRContext(N, Nc::Integer, Nt::Integer, K::Integer, patch_sizes, strides;
                     form::Symbol=:tuned)
    length(patch_sizes) == length(strides) ||
        throw(ArgumentError("patch_sizes and strides differ in length"))
    ps = Int32[p for s in patch_sizes for p in s]
    ss = Int32[p for s in strides for p in s]
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:mslr_create, libmslr), Cint,
               (Ptr{Int32}, Int32, Int32, Int64, Int32, Ptr{Int32}, Ptr{Int32}, Int32,
                Ptr{Ptr{Cvoid}}),
               Int32[N...], Nc, Nt, K, length(patch_sizes), ps, ss,
               form === :tuned ? FORM_TUNED : form === :tf32 ? FORM_TF32 : FORM_PLAIN, out)
    _check(rc)
    ctx = MSLRContext(out[], Tuple(Int.(N)), Int(Nc), Int(Nt), Int(K), length(patch_sizes), 0)
    finalizer(close, ctx)
    return ctx
end

function Base.close(ctx::MSLRContext)
    if ctx.h != C_NULL
        ccall((:mslr_destroy, libmslr), Cint, (Ptr{Cvoid},), ctx.h)
        ctx.h = C_NULL
    end
    return nothing
end

"""
    bind!(ctx, smaps, ksp, idx)

Bind the acquisition: SOS-normalised coil maps `(Nx,Ny,Nz,Nc)`, k-space
`(K,Nc,Nt)` and 1-based sample indices `(K,Nt)` (`findall(vec(Ω_t))` per
frame, scripts/reconstruct.jl:144-147).  The library keeps its own copies.
"""
function bind!(ctx::MSLRContext, smaps::CuArray{ComplexF32}, ksp::CuArray{ComplexF32},
               idx::CuArray{Int32})
    size(smaps) == (ctx.N..., ctx.Nc) || throw(ArgumentError("smaps size $(size(smaps))"))
    size(ksp) == (ctx.K, ctx.Nc, ctx.Nt) || throw(ArgumentError("ksp size $(size(ksp))"))
    size(idx) == (ctx.K, ctx.Nt) || throw(ArgumentError("idx size $(size(idx))"))
    _check(ccall((:mslr_bind, libmslr), Cint,
                 (Ptr{Cvoid}, CuPtr{ComplexF32}, CuPtr{ComplexF32}, CuPtr{Int32}, Int32, Ptr{Cvoid}),
                 ctx.h, smaps, ksp, idx, Int32(1), _stream()), ctx.h)
    return ctx
end

"""A * x over all frames (Asense_gpu fwd per frame, block_diag)."""
function sense_forward!(y::CuArray{ComplexF32}, ctx::MSLRContext, x::CuArray{ComplexF32})
    _check(ccall((:mslr_sense_forward, libmslr), Cint,
                 (Ptr{Cvoid}, CuPtr{ComplexF32}, CuPtr{ComplexF32}, Ptr{Cvoid}),
                 ctx.h, x, y, _stream()), ctx.h)
    return y
end

"""A' * y (exact unitary adjoint, src/sense_gpu.jl:84-101)."""
function sense_adjoint!(x::CuArray{ComplexF32}, ctx::MSLRContext, y::CuArray{ComplexF32})
    _check(ccall((:mslr_sense_adjoint, libmslr), Cint,
                 (Ptr{Cvoid}, CuPtr{ComplexF32}, CuPtr{ComplexF32}, Ptr{Cvoid}),
                 ctx.h, y, x, _stream()), ctx.h)
    return x
end

"""
    dc_cost_grad!(g, ctx, X)

`A'(A Σ_k X[..,k] − y)` into `g` `(Nx,Ny,Nz,Nt)`; the reference then
`repeat`s it over the scales (scripts/reconstruct.jl:180-183).
"""
function dc_cost_grad!(g::CuArray{ComplexF32}, ctx::MSLRContext, X::CuArray{ComplexF32})
    _check(ccall((:mslr_normal_op, libmslr), Cint,
                 (Ptr{Cvoid}, CuPtr{ComplexF32}, Int32, CuPtr{ComplexF32}, Int32, Ptr{Cvoid}),
                 ctx.h, X, Int32(size(X, 5)), g, Int32(1), _stream()), ctx.h)
    return g
end

"""
    patch_svst!(out, ctx, img, k, β)

`patchSVST_gpu(img, β, PATCH_SIZES[k], STRIDES[k])` for scale `k` (1-based)
into `out` (may be `img`: the reference's g_prox writes in place).
"""
function patch_svst!(out::CuArray{ComplexF32}, ctx::MSLRContext, img::CuArray{ComplexF32},
                     k::Integer, β::Real)
    _check(ccall((:mslr_patch_svst, libmslr), Cint,
                 (Ptr{Cvoid}, Int32, Float64, CuPtr{ComplexF32}, CuPtr{ComplexF32}, Ptr{Cvoid}),
                 ctx.h, Int32(k - 1), Float64(β), img, out, _stream()), ctx.h)
    return out
end

"""
    pogm_run!(ctx, X, niter, L; restart_cutoff=0.0, bsig=1.0, costs=false)

`pogm_mod(X, ..., dc_cost_grad, L; mom=:pogm, restart=:gr, niter, g_prox)`
with run_recon's closures, overwriting `X` `(Nx,Ny,Nz,Nt,Ns)`.  Returns the
per-iteration restart flags (entry 1 is false, as the logger's first entry).
With `costs=true` it returns `(dc_costs, reg_costs, restarts)`, the three
vectors run_recon's logger collects and saves
(scripts/reconstruct.jl:204-205, :228-230): the costs of X0 and of every
iterate, FP64.
"""
function pogm_run!(ctx::MSLRContext, X::CuArray{ComplexF32}, niter::Integer, L::Real;
                   restart_cutoff::Real=0.0, bsig::Real=1.0, costs::Bool=false)
    flags = zeros(UInt8, niter + 1)
    if costs
        dc = zeros(Float64, niter + 1)
        reg = zeros(Float64, niter + 1)
        _check(ccall((:mslr_pogm_run_costs, libmslr), Cint,
                     (Ptr{Cvoid}, CuPtr{ComplexF32}, Int32, Float64, Float64, Float64, Ptr{UInt8},
                      Ptr{Float64}, Ptr{Float64}, Ptr{Cvoid}),
                     ctx.h, X, Int32(niter), Float64(L), Float64(restart_cutoff), Float64(bsig),
                     flags, dc, reg, _stream()), ctx.h)
        return dc, reg, Bool.(flags)
    end
    _check(ccall((:mslr_pogm_run, libmslr), Cint,
                 (Ptr{Cvoid}, CuPtr{ComplexF32}, Int32, Float64, Float64, Float64, Ptr{UInt8},
                  Ptr{Cvoid}),
                 ctx.h, X, Int32(niter), Float64(L), Float64(restart_cutoff), Float64(bsig),
                 flags, _stream()), ctx.h)
    return Bool.(flags)
end

"""
    pogm_mod!(ctx, X, niter, L; mom=:pogm, restart=:gr, f_mu=0.0, restart_cutoff=0.0, bsig=1.0)

`pogm_mod` (src/mirt_mod.jl:74-188) with any of its options and run_recon's
closures, from `X` (x0) in place: `X` receives `xnew` for `:pogm`, `ynew` for
`:pgm` / `:fpgm`.  `restart=:fr` uses run_recon's comp_cost.  Throws
`ArgumentError` for an unknown `mom` / `restart`, as pogm_mod does.  Returns
the restart flags (entry 1 is false).
"""
function pogm_mod!(ctx::MSLRContext, X::CuArray{ComplexF32}, niter::Integer, L::Real;
                   mom::Symbol=:pogm, restart::Symbol=:gr, f_mu::Real=0.0,
                   restart_cutoff::Real=0.0, bsig::Real=1.0)
    m = Dict(:pgm => 0, :fpgm => 1, :pogm => 2)
    r = Dict(:none => 0, :gr => 1, :fr => 2)
    haskey(m, mom) || throw(ArgumentError("mom=$mom"))
    haskey(r, restart) || throw(ArgumentError("restart=$restart"))
    flags = zeros(UInt8, niter + 1)
    _check(ccall((:mslr_pogm_run_options, libmslr), Cint,
                 (Ptr{Cvoid}, CuPtr{ComplexF32}, Int32, Float64, Float64, Int32, Int32, Float64,
                  Float64, Ptr{UInt8}, Ptr{Cvoid}),
                 ctx.h, X, Int32(niter), Float64(L), Float64(f_mu), Int32(m[mom]), Int32(r[restart]),
                 Float64(restart_cutoff), Float64(bsig), flags, _stream()), ctx.h)
    return Bool.(flags)
end

"""
    cost(ctx, X) -> (dc_cost, reg_cost)

The two terms of run_recon's cost for `X` `(Nx,Ny,Nz,Nt,Ns)`
(scripts/reconstruct.jl:176-194): ½‖A Σ_k X[..,k] − y‖² and
Σ_k λ_k patch_nucnorm(img2patches(X[..,k])), FP64.
"""
function cost(ctx::MSLRContext, X::CuArray{ComplexF32})
    dc = Ref{Float64}(0.0)
    reg = Ref{Float64}(0.0)
    _check(ccall((:mslr_cost, libmslr), Cint,
                 (Ptr{Cvoid}, CuPtr{ComplexF32}, Int32, Ref{Float64}, Ref{Float64}, Ptr{Cvoid}),
                 ctx.h, X, Int32(size(X, 5)), dc, reg, _stream()), ctx.h)
    return dc[], reg[]
end

"""
    sync!(ctx)

Wait for the context's work on the task-local stream and raise any error its
kernels recorded since the last check (a bounded wait that ran out, a
non-finite restart sum) — the asynchronous calls (`dc_cost_grad!`,
`patch_svst!`, the operators) leave those to the next synchronising call.
"""
function sync!(ctx::MSLRContext)
    _check(ccall((:mslr_sync, libmslr), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), ctx.h, _stream()), ctx.h)
    return ctx
end

"""X0 of scripts/reconstruct.jl:209-214: X[..,1] = A'y, other scales 0."""
function init_x0!(ctx::MSLRContext, X::CuArray{ComplexF32})
    _check(ccall((:mslr_init_x0, libmslr), Cint, (Ptr{Cvoid}, CuPtr{ComplexF32}, Ptr{Cvoid}),
                 ctx.h, X, _stream()), ctx.h)
    return X
end

"""σ₁(A) by poweriter_mod (src/mirt_mod.jl:215-238), x0 = ones."""
function power_iter(ctx::MSLRContext; niter::Integer=200, tol::Real=1e-6)
    s1 = Ref{Float64}(0.0)
    it = Ref{Int32}(0)
    _check(ccall((:mslr_power_iter, libmslr), Cint,
                 (Ptr{Cvoid}, Int32, Float64, Ref{Float64}, Ref{Int32}, Ptr{Cvoid}),
                 ctx.h, Int32(niter), Float64(tol), s1, it, _stream()), ctx.h)
    return s1[], Int(it[])
end

"""
    set_lambdas!(ctx, λs)

Per-scale weights λ_k of g_prox (`c * λs[k]`, scripts/reconstruct.jl:196-202);
the context starts from the Ong–Lustig values of :164-169.
"""
function set_lambdas!(ctx::MSLRContext, λs::AbstractVector{<:Real})
    length(λs) == ctx.Ns || throw(ArgumentError("need $(ctx.Ns) lambdas"))
    _check(ccall((:mslr_set_lambdas, libmslr), Cint, (Ptr{Cvoid}, Ptr{Float64}),
                 ctx.h, Float64.(collect(λs))), ctx.h)
    return ctx
end

"""
    pogm_grad(ctx, X_true, niter, L; restart_cutoff=0.0, bsig=1.0) -> (loss, ∂loss/∂log λ, X, restarts)

Runs `pogm_run!`'s iteration for `niter` steps from X0 = A'y and returns
loss = ½‖Σ_k X[..,k] − X_true‖² (X_true `(Nx,Ny,Nz,Nt)`), its gradient with
respect to log λ_k (reverse accumulation through the SENSE normal operator
and the patch-SVST backward, restart decisions held fixed), the final X and
the restart flags.
"""
function pogm_grad(ctx::MSLRContext, X_true::CuArray{ComplexF32}, niter::Integer, L::Real;
                   restart_cutoff::Real=0.0, bsig::Real=1.0)
    size(X_true) == (ctx.N..., ctx.Nt) || throw(ArgumentError("X_true size $(size(X_true))"))
    X = CuArray{ComplexF32}(undef, ctx.N..., ctx.Nt, ctx.Ns)
    loss = Ref{Float64}(0.0)
    grad = zeros(Float64, ctx.Ns)
    flags = zeros(UInt8, niter + 1)
    _check(ccall((:mslr_pogm_grad, libmslr), Cint,
                 (Ptr{Cvoid}, CuPtr{ComplexF32}, Int32, Float64, Float64, Float64, CuPtr{ComplexF32},
                  Ref{Float64}, Ptr{Float64}, Ptr{UInt8}, Ptr{Cvoid}),
                 ctx.h, X_true, Int32(niter), Float64(L), Float64(restart_cutoff), Float64(bsig), X,
                 loss, grad, flags, _stream()), ctx.h)
    return loss[], grad, X, Bool.(flags)
end

"""
    mslr_sampling(N, Nc, Nt, ksp0) -> K

Samples per frame of the zero-filled k-space `ksp0` `(Nx,Ny,Nz,Nc,Nt)`: the
mask Ω = ksp0[:,:,:,1,:] .!= 0 with the checks of scripts/reconstruct.jl:113-118
(`ArgumentError` with the reference's messages otherwise).
"""
function mslr_sampling(N, Nc::Integer, Nt::Integer, ksp0::CuArray{ComplexF32})
    K = Ref{Int64}(0)
    _check(ccall((:mslr_sampling, libmslr), Cint,
                 (Ptr{Int32}, Int32, Int32, CuPtr{ComplexF32}, Ref{Int64}, Ptr{Int32}, Ptr{Cvoid},
                  Int64, Ptr{Cvoid}),
                 Int32[N...], Int32(Nc), Int32(Nt), ksp0, K, C_NULL, C_NULL, Int64(0), _stream()))
    return Int(K[])
end

"""
    prepare!(ctx, ksp0, smaps_raw) -> (smaps, ksp, idx, scale_factor)

scripts/reconstruct.jl:86-147 on the device: SOS-normalised maps, the samples
`(K,Nc,Nt)` divided by quantile(abs.(sense_comb(ksp0, smaps)), 0.99), the
0-based sample indices `(K,Nt)`; the context is bound to them.
"""
function prepare!(ctx::MSLRContext, ksp0::CuArray{ComplexF32}, smaps_raw::CuArray{ComplexF32})
    smaps = similar(smaps_raw)
    ksp = CuArray{ComplexF32}(undef, ctx.K, ctx.Nc, ctx.Nt)
    idx = CuArray{Int32}(undef, ctx.K, ctx.Nt)
    sf = Ref{Float64}(0.0)
    _check(ccall((:mslr_prepare, libmslr), Cint,
                 (Ptr{Cvoid}, CuPtr{ComplexF32}, CuPtr{ComplexF32}, CuPtr{ComplexF32}, CuPtr{ComplexF32},
                  CuPtr{Int32}, Ref{Float64}, Ptr{Cvoid}),
                 ctx.h, ksp0, smaps_raw, smaps, ksp, idx, sf, _stream()), ctx.h)
    return smaps, ksp, idx, sf[]
end

"""Time the free launch shapes on the bound context and keep the fastest."""
function autotune!(ctx::MSLRContext)
    _check(ccall((:mslr_autotune, libmslr), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), ctx.h, _stream()), ctx.h)
    return ctx
end

"""Ong–Lustig λ_k of scripts/reconstruct.jl:164-169."""
function mslr_lambdas(N, Nt::Integer, patch_sizes)
    return [sqrt(prod(ps)) + sqrt(Nt) + sqrt(log(prod(N) * Nt / max(prod(ps), Nt)))
            for ps in patch_sizes]
end

end # module
