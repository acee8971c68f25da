/*
 * mslr.h — C ABI of the B200 (sm_100a) MSLR hot-path library, libmslr.so.
 *
 * Replaces, for one GPU, the per-iteration path of rextlfung/mslr-recon:
 *   - the SENSE operator            src/sense_gpu.jl:56-108   (Asense_gpu fwd/adj)
 *   - the data-consistency gradient scripts/reconstruct.jl:180-183 (dc_cost_grad)
 *   - patch SVST with extract/recombine
 *                                   src/recon.jl:53-126, :183-269,
 *                                   src/sense_gpu.jl:122-223 (patchSVST_gpu)
 *   - POGM with gradient restart    src/mirt_mod.jl:26-29, :74-188 (pogm_mod)
 *   - power iteration               src/mirt_mod.jl:215-238 (poweriter_mod)
 *   - run_recon's closures and X0   scripts/reconstruct.jl:159-214
 *
 * Conventions (those of the reference's Julia arrays):
 *   - complex data are interleaved float pairs (ComplexF32), column-major:
 *       image        (Nx, Ny, Nz, Nt)          X (Nx, Ny, Nz, Nt, Ns)
 *       coil maps    (Nx, Ny, Nz, Nc)          k-space y (K, Nc, Nt)
 *       patch stack  (p, Nt, Np)
 *     so x is the fastest index everywhere;
 *   - sample indices idx (K, Nt) are int32 linear indices into the centred
 *     (Nx, Ny, Nz) k-space grid, ascending per frame — the reference's
 *     findall(vec(samp)) — 1-based when index_base == 1, 0-based when 0;
 *   - every device pointer is BORROWED: the library never frees caller
 *     memory; all workspaces are owned by the context and allocated in
 *     mslr_create / mslr_bind, never inside the per-iteration calls;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default);
 *   - every call returns an int status (MSLR_OK == 0) and never aborts;
 *     mslr_last_error() returns a message for the last failure on a context
 *     (or, with ctx == NULL, for the calling thread's last context-free call);
 *   - one context must not be used from two host threads at once.
 */
#ifndef MSLR_H
#define MSLR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MSLR_ABI_VERSION 1

#define MSLR_OK 0
#define MSLR_ERR_ARG 1           /* bad shape, pointer or value (ArgumentError / @assert) */
#define MSLR_ERR_CUDA 2          /* a CUDA runtime call failed */
#define MSLR_ERR_STATE 3         /* call out of order (e.g. before mslr_bind) */
#define MSLR_ERR_UNSUPPORTED 4   /* shape outside what the kernels support */
#define MSLR_ERR_NONFINITE 5     /* NaN/Inf met in a reduction */
#define MSLR_ERR_NOMEM 6         /* device allocation failed */

/* Computation forms (mslr_create `form`). */
#define MSLR_FORM_PLAIN 0        /* FP32 SIMT Gram/rebuild, one launch sequence per scale, no graph */
#define MSLR_FORM_TUNED 1        /* split-precision tensor-core Gram/rebuild, graph-captured iteration */
#define MSLR_FORM_TF32 2         /* as TUNED with TF32 (not split) tensor-core Gram/rebuild products */

/* pogm_mod's `mom` and `restart` options (mslr_pogm_run_options). */
#define MSLR_MOM_PGM 0           /* :pgm  — proximal gradient */
#define MSLR_MOM_FPGM 1          /* :fpgm — FISTA momentum */
#define MSLR_MOM_POGM 2          /* :pogm — optimised gradient (run_recon's choice) */
#define MSLR_RESTART_NONE 0      /* :none */
#define MSLR_RESTART_GR 1        /* :gr — gradient restart (run_recon's choice) */
#define MSLR_RESTART_FR 2        /* :fr — function restart on comp_cost = dc_cost + reg_cost */

typedef struct mslr_ctx mslr_ctx;

/* Library ABI version (MSLR_ABI_VERSION). */
int mslr_abi_version(void);

/* Last error message for `ctx` (ctx == NULL: the calling thread's last
 * context-free error).  The string stays valid until the next failing call. */
const char* mslr_last_error(const mslr_ctx* ctx);

/* ------------------------------------------------------------------------
 * Patch geometry (host only) — src/recon.jl:54-72.
 * For one scale: clamps ps to N, nsteps[d] = cld(N[d]-ps[d], ss[d]),
 * Np = prod(nsteps+1).  `starts` (optional, may be NULL) receives the
 * 0-based patch starts of each dimension concatenated:
 * (nsteps[0]+1) x-starts, then y-starts, then z-starts.
 * ------------------------------------------------------------------------ */
int mslr_patch_geometry(const int32_t N[3], const int32_t patch[3], const int32_t stride[3],
                        int32_t ps_out[3], int32_t nsteps_out[3], int64_t* Np_out,
                        int32_t* starts);

/* img2patches (src/recon.jl:53-78; src/sense_gpu.jl:168-192):
 * img (Nx,Ny,Nz,Nt) -> P (p, Nt, Np), device pointers. */
int mslr_img2patches(const int32_t N[3], int32_t Nt, const int32_t patch[3],
                     const int32_t stride[3], const void* img, void* P, void* stream);

/* patches2img (src/recon.jl:96-126; src/sense_gpu.jl:194-223):
 * P (p, Nt, Np) -> img (Nx,Ny,Nz,Nt): patch sums in ascending ip divided by
 * max(coverage count, 1). */
int mslr_patches2img(const int32_t N[3], int32_t Nt, const int32_t patch[3],
                     const int32_t stride[3], const void* P, void* img, void* stream);

/* ------------------------------------------------------------------------
 * Batched SVST (src/recon.jl:183-211 SVST; src/sense_gpu.jl:122-128 SVST_gpu)
 * on `batch` independent m x n column-major complex matrices stored back to
 * back: out_b = U diag(max(S - beta_b, 0)) V^H, zero when ||A_b|| == 0.
 * `betas` is a host array of `batch` thresholds.  The caller provides device
 * scratch of at least mslr_svst_batch_workspace() bytes.  in may equal out.
 * Synchronises `stream` and reads the call's device error word: when a
 * tensor-core kernel's bounded wait ran out (mslr_set_wait_limit) the call
 * returns MSLR_ERR_CUDA and `out` is not valid.
 * ------------------------------------------------------------------------ */
int mslr_svst_batch_workspace(int32_t m, int32_t n, int32_t batch, size_t* bytes);
int mslr_svst_batch(int32_t m, int32_t n, int32_t batch, const double* betas,
                    const void* in, void* out, void* workspace, size_t workspace_bytes,
                    int32_t form, void* stream);

/* Size of the fixed scratch array behind mslr_svst_batch_noalloc (16 MiB). */
#define MSLR_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)

/* Batched SVST that allocates nothing.  No counterpart in the reference: it
 * exists for callers that cannot call cudaMalloc — e.g. a host framework
 * whose memory pool owns the device (Julia's CUDA.jl or PyTorch's caching
 * allocator) and must not have a library allocate behind the pool, or a
 * real-time pipeline running on a fixed memory plan.  Same arguments and
 * results as mslr_svst_batch, but the scratch is a file-scope device array
 * of MSLR_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds
 * until the process exits.  A batch needing more scratch than that
 * (mslr_svst_batch_workspace reports the need) is rejected with
 * MSLR_ERR_ARG.  The first call on each device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture.  All calls share the one array, so calls
 * that overlap on the GPU (different streams, or different host threads
 * without ordering) race and corrupt each other's results.  Like
 * mslr_svst_batch it synchronises `stream` and reports a timed-out bounded
 * wait as MSLR_ERR_CUDA (its error word lives in the fixed array too). */
int mslr_svst_batch_noalloc(int32_t m, int32_t n, int32_t batch, const double* betas,
                            const void* in, void* out, void* stream);

/* ------------------------------------------------------------------------
 * Reconstruction context — the state run_recon builds
 * (scripts/reconstruct.jl:133-214) for Ns scales of patch sizes/strides.
 * patch/stride: 3*n_scales int32 (x,y,z per scale).  K = samples per frame
 * (uniform across frames, scripts/reconstruct.jl:116-118).
 * ------------------------------------------------------------------------ */
int mslr_create(const int32_t N[3], int32_t Nc, int32_t Nt, int64_t K, int32_t n_scales,
                const int32_t* patch, const int32_t* stride, int32_t form, mslr_ctx** out);
int mslr_destroy(mslr_ctx* ctx);

/* Device bytes the context holds (after create / bind). */
int mslr_workspace_bytes(const mslr_ctx* ctx, size_t* bytes);

/* Bind the acquisition: coil maps smaps (Nx,Ny,Nz,Nc), k-space y (K,Nc,Nt),
 * indices idx (K,Nt).  The library keeps its own device copies of what it
 * needs (modulated maps, per-frame sampling bitmasks, indices, A'y), so the
 * caller may free its buffers afterwards.  Validates that indices are in
 * range and strictly ascending per frame (MSLR_ERR_ARG otherwise). */
int mslr_bind(mslr_ctx* ctx, const void* smaps, const void* y, const int32_t* idx,
              int32_t index_base, void* stream);

/* Asense forward over all frames (src/sense_gpu.jl:71-81 per frame,
 * block_diag at scripts/reconstruct.jl:142): x (Nx,Ny,Nz,Nt) -> y (K,Nc,Nt). */
int mslr_sense_forward(mslr_ctx* ctx, const void* x, void* y, void* stream);

/* Exact unitary adjoint (src/sense_gpu.jl:84-101 with scale*bfft):
 * y (K,Nc,Nt) -> x (Nx,Ny,Nz,Nt). */
int mslr_sense_adjoint(mslr_ctx* ctx, const void* y, void* x, void* stream);

/* dc_cost_grad before the repeat (scripts/reconstruct.jl:180-183):
 * g = A'(A * sum_k X[..,k] - y) for X (Nx,Ny,Nz,Nt,ns_in); with
 * subtract_data == 0, g = A'A * sum_k X[..,k]. */
int mslr_normal_op(mslr_ctx* ctx, const void* X, int32_t ns_in, void* g,
                   int32_t subtract_data, void* stream);

/* Profiling hook (no counterpart in the reference): runs mslr_normal_op with
 * subtract_data = 1 once, recording CUDA events on `stream` around every
 * kernel of every chunk, and returns in kernel_ms[0..3] the average device
 * time per launch of the chunk's kernels and in launches_per_kernel[0..3]
 * their launch counts.  Four-pass form (the default): [0] forward plane pass
 * (coil maps × summed image, DFT_y, DFT_x), [1] z pass with the k-space mask,
 * [2] inverse plane pass with × conj(coil map), [3] coil combine.  Three-kernel
 * form (MSLR_SENSE_PATH=3, or the tensor-core plane pass): [0] forward z pass,
 * [1] plane pass, [2] adjoint z pass with the coil combine, [3] zero.  Both
 * arrays must hold 4 entries.  Synchronises `stream`.  MSLR_ERR_UNSUPPORTED
 * unless the tuned form runs the shape-specialised SENSE kernels for this
 * image shape. */
int mslr_normal_op_profile(mslr_ctx* ctx, const void* X, int32_t ns_in, void* g, void* stream,
                           double* kernel_ms, int64_t* launches_per_kernel);

/* patchSVST for scale `scale` (0-based) with global threshold beta
 * (src/recon.jl:251-256; src/sense_gpu.jl:138-145): img_in (Nx,Ny,Nz,Nt)
 * -> img_out.  img_in may equal img_out. */
int mslr_patch_svst(mslr_ctx* ctx, int32_t scale, double beta, const void* img_in,
                    void* img_out, void* stream);

/* patchSVST with one threshold per patch (src/recon.jl:263-268;
 * src/sense_gpu.jl:153-160): `lambdas` is a host array of the scale's Np
 * thresholds (patch order of mslr_patch_geometry), used as β of each patch.
 * img_in may equal img_out. */
int mslr_patch_svst_lambdas(mslr_ctx* ctx, int32_t scale, const double* lambdas, const void* img_in,
                            void* img_out, void* stream);

/* patch_nucnorm of scale `scale`'s patches of img (Nx,Ny,Nz,Nt): with
 * lambdas == NULL Σ_patches Σσ (src/recon.jl:138-146); with a host array of
 * Np weights, Σ_patches λ_p Σσ_p / Np (src/recon.jl:154-166).  FP64 sums in
 * patch order; the singular values come from each patch Gram's eigenvalues.
 * Synchronises `stream`. */
int mslr_patch_nucnorm(mslr_ctx* ctx, int32_t scale, const double* lambdas, const void* img, double* cost,
                       void* stream);

/* The two terms of run_recon's cost (scripts/reconstruct.jl:176-194,
 * logged each iteration by its logger, :205) for X (Nx,Ny,Nz,Nt,ns_in):
 *   dc_cost  = ½ ‖A Σ_k X[..,k] − y‖²
 *   reg_cost = Σ_k λ_k · patch_nucnorm(img2patches(X[..,k]))  (ns_in == n_scales)
 * FP64 sums.  dc_cost is formed from one normal operator, A'y and ‖y‖²
 * (kept from bind); reg_cost from the eigenvalues of every patch's Gram
 * matrix.  Either output pointer may be NULL.  Synchronises `stream`. */
int mslr_cost(mslr_ctx* ctx, const void* X, int32_t ns_in, double* dc_cost, double* reg_cost,
              void* stream);

/* X0 of scripts/reconstruct.jl:209-214: X[..,1] = A'y, other scales 0. */
int mslr_init_x0(mslr_ctx* ctx, void* X, void* stream);

/* pogm_mod (src/mirt_mod.jl:74-188) with mom=:pogm, restart=:gr and
 * run_recon's closures (scripts/reconstruct.jl:180-202), starting from and
 * overwriting X (Nx,Ny,Nz,Nt,Ns).  L is the Lipschitz constant
 * (Ns*sigma1^2).  restarts_host (optional, length niter+1) receives the
 * per-iteration restart flags (entry 0 is false, as the logger's out[1]).
 * The reference's in-place g_prox makes xnew alias znew; this recurrence is
 * reproduced exactly. */
int mslr_pogm_run(mslr_ctx* ctx, void* X, int32_t niter, double L, double restart_cutoff,
                  double bsig, uint8_t* restarts_host, void* stream);

/* As mslr_pogm_run, and also fills run_recon's logged costs
 * (scripts/reconstruct.jl:204-205, saved at :228-230): dc_costs_host[i] and
 * reg_costs_host[i] (host arrays of niter+1, either may be NULL) receive
 * mslr_cost's dc_cost and reg_cost of X0 (i = 0) and of x_i after iteration i.
 * Synchronises `stream` once per iteration. */
int mslr_pogm_run_costs(mslr_ctx* ctx, void* X, int32_t niter, double L, double restart_cutoff,
                        double bsig, uint8_t* restarts_host, double* dc_costs_host,
                        double* reg_costs_host, void* stream);

/* pogm_mod (src/mirt_mod.jl:74-188) with any of its options and run_recon's
 * closures: mom (MSLR_MOM_*), restart (MSLR_RESTART_*), f_mu = mu >= 0.  For
 * :fr, Fcost is run_recon's comp_cost (dc_cost + reg_cost, as mslr_cost).
 * On return X holds pogm_mod's result: x_niter for :pogm, y_niter for :pgm
 * and :fpgm.  Argument errors as src/mirt_mod.jl:88-93 (MSLR_ERR_ARG).
 * mom = :pogm, restart = :gr, mu = 0 is mslr_pogm_run (the graph-replayed
 * iteration); every other combination runs a host-driven loop that
 * synchronises `stream` once or twice per iteration, and :pgm / :fpgm
 * allocate one more (Ns, Nt, nvox) buffer on first use. */
int mslr_pogm_run_options(mslr_ctx* ctx, void* X, int32_t niter, double L, double mu, int32_t mom,
                          int32_t restart, double restart_cutoff, double bsig, uint8_t* restarts_host,
                          void* stream);

/* Stepwise POGM: mslr_pogm_begin sets up the state for `niter` iterations
 * from X; each mslr_pogm_step runs exactly one iteration (X holds x_i
 * after it returns, stream-ordered).  mslr_pogm_step does not synchronise:
 * a device-side error of its kernels (a timed-out bounded wait, a
 * non-finite restart sum) is reported by the next synchronising call on the
 * context — mslr_pogm_restarts, mslr_sync, mslr_pogm_run. */
int mslr_pogm_begin(mslr_ctx* ctx, void* X, int32_t niter, double L, double restart_cutoff,
                    double bsig, void* stream);
int mslr_pogm_step(mslr_ctx* ctx, void* X, void* stream);

/* Tuned and TF32 forms: capture the POGM iteration into a CUDA graph on first use
 * and replay it (enable = 1, the default), or launch its kernels directly
 * (enable = 0).  Both give bit-identical results. */
int mslr_set_graph(mslr_ctx* ctx, int32_t enable);
/* Restart flags of the iterations run so far (host array of niter+1).
 * Synchronises `stream` and reports pending device-side errors as mslr_sync. */
int mslr_pogm_restarts(mslr_ctx* ctx, uint8_t* restarts_host, void* stream);

/* Device-side errors (no counterpart in the reference, whose CUDA.jl calls
 * throw).  Kernels of a context record errors in the context's own device
 * error word instead of aborting: MSLR_ERR_NONFINITE for a NaN/Inf restart
 * sum, MSLR_ERR_CUDA for a bounded wait that ran out (the results written
 * since the previous check are then not valid).  mslr_sync synchronises
 * `stream`, reads and clears the word and returns the matching status;
 * mslr_pogm_run, mslr_pogm_run_costs, mslr_pogm_grad, mslr_pogm_restarts,
 * mslr_cost, mslr_power_iter and mslr_normal_op_profile do the same before
 * they return.  The asynchronous entries (mslr_normal_op, mslr_patch_svst,
 * mslr_pogm_step, the SENSE operators) leave their errors to the next such
 * call. */
int mslr_sync(mslr_ctx* ctx, void* stream);

/* Poll count after which a tensor-core kernel's bounded mbarrier wait gives
 * up (default 2^22, a few tens of milliseconds).  ctx == NULL sets it for the
 * context-free mslr_svst_batch / mslr_svst_batch_noalloc calls of the whole
 * process.  A kernel whose wait gives up still waits (with the default
 * count) for the work it already issued, writes its output tile as zeros,
 * frees its tensor memory and returns; the call then reports MSLR_ERR_CUDA.
 * A small value exists to test that path; 0 makes every such wait give up. */
int mslr_set_wait_limit(mslr_ctx* ctx, int64_t polls);

/* ------------------------------------------------------------------------
 * Sharded iteration over several GPUs (no counterpart in the reference, which
 * runs on one device).  One process per GPU; each rank holds a context for
 * its block of frames (the SENSE normal operator and the POGM state) and a
 * context for its z-slab of the volume (patch SVST over all frames).  Per
 * iteration (mslr-recon_b200/sharded.py drives it over torch.distributed):
 *   mslr_pogm_step_local   g = A'(A Σ_k x_k − y) on the rank's frames, the
 *                          momentum scalars, u, and z into Z (Ns, Nt_rank,
 *                          nvox); the rank's restart totals into sums_dev
 *                          (4 doubles on the device: Σ Re(−g·Δu), Σ|g|²,
 *                          Σ|Δu|², Σ Re(g·gold)) — no decision yet;
 *   (the caller sums sums_dev over the ranks)
 *   mslr_pogm_step_decide  the restart decision and t/σ update from the
 *                          totals (src/mirt_mod.jl:163-184), identical on
 *                          every rank;
 *   mslr_pogm_scalars      α, β, γ, ζ of the iteration to the host
 *                          (synchronises `stream`): the caller's thresholds
 *                          are ζ·λ_k;
 *   (the caller moves z from frames to slabs, all-to-all)
 *   mslr_patch_svst        on the slab for a scale that tiles it;
 *   mslr_patch_gram        for the global patch: the slab's partial Gram
 *                          (n × n, column-major; a tall patch's Gram Pᴴ P is
 *                          a sum over voxels), summed over the ranks by the
 *                          caller, then
 *   mslr_patch_svst_gram   SVST of the slab's rows of that patch from the
 *                          summed Gram (eigen stage, W, rebuild);
 *   (the caller moves x from slabs back to frames, all-to-all).
 * mslr_patch_gram / mslr_patch_svst_gram need a single-patch scale.
 * ------------------------------------------------------------------------ */
int mslr_pogm_step_local(mslr_ctx* ctx, void* X, void* Z, double* sums_dev, void* stream);
int mslr_pogm_step_decide(mslr_ctx* ctx, const double* sums_dev, void* stream);
int mslr_pogm_scalars(mslr_ctx* ctx, double* alpha_beta_gamma_zeta, void* stream);
int mslr_patch_gram(mslr_ctx* ctx, int32_t scale, const void* img, void* gram, void* stream);
int mslr_patch_svst_gram(mslr_ctx* ctx, int32_t scale, double beta, const void* gram, const void* img_in,
                         void* img_out, void* stream);

/* Set-up of run_recon's inputs on the device (scripts/reconstruct.jl:86-147).
 *
 * mslr_sos_normalize: smaps_out = S ./ (sqrt.(sum(abs2.(S); dims=4)) .+ eps(Float32))
 *   for raw coil maps S (Nx,Ny,Nz,Nc) (:89), Float32, coils summed in order.
 *   smaps_out may equal smaps_raw.
 * mslr_sampling: the sampling mask Ω = ksp[:,:,:,1,:] .!= 0 of the zero-filled
 *   k-space ksp (Nx,Ny,Nz,Nc,Nt) and the checks of :109-118 — every coil has
 *   coil 1's pattern, every frame the same count (MSLR_ERR_ARG with the
 *   reference's messages otherwise).  *K receives the samples per frame; with
 *   idx / y non-NULL (capacity K_cap per frame) it also gathers the 0-based
 *   ascending indices idx (K, Nt) and the samples y (K, Nc, Nt) (:144-147).
 * mslr_prepare: on a context created with that K — normalised maps into
 *   smaps_out, idx and the samples gathered, bound, then the scale factor
 *   quantile(abs.(sense_comb(ksp, smaps)), 0.99) (:100-104, src/recon.jl:310-321;
 *   type-7 quantile, exact order statistics) into *scale_factor, y divided by
 *   max(scale, eps(Float32)) in place and the context bound to it.  The mask
 *   is taken before the division; a sample that the division turns into zero
 *   is reported as MSLR_ERR_ARG.  Synchronises `stream`. */
int mslr_sos_normalize(const int32_t N[3], int32_t Nc, const void* smaps_raw, void* smaps_out,
                       void* stream);
int mslr_sampling(const int32_t N[3], int32_t Nc, int32_t Nt, const void* ksp, int64_t* K, int32_t* idx,
                  void* y, int64_t K_cap, void* stream);
int mslr_prepare(mslr_ctx* ctx, const void* ksp, const void* smaps_raw, void* smaps_out, void* y_out,
                 int32_t* idx_out, double* scale_factor, void* stream);

/* Per-scale regularisation weights λ_k (scripts/reconstruct.jl:164-169 computes
 * them by the Ong–Lustig formula; mslr_create starts from those values).
 * The threshold of scale k in g_prox is ζ·λ_k (scripts/reconstruct.jl:196-202). */
int mslr_set_lambdas(mslr_ctx* ctx, const double* lambdas);
int mslr_get_lambdas(const mslr_ctx* ctx, double* lambdas);

/* Gradient of the unrolled POGM.  Runs niter iterations of mslr_pogm_run's
 * recurrence from X0 = A'y (scripts/reconstruct.jl:209-226; X receives
 * x_niter) and returns loss = ½‖Σ_k X[..,k] − X_true‖² (X_true
 * (Nx,Ny,Nz,Nt), FP64 sum) and grad_loglam[k] = d loss / d log λ_k, by
 * reverse accumulation through the SENSE normal operator and the patch-SVST
 * backward, with z_i stored per iteration and each patch's eigen-
 * decomposition recomputed.  Restart decisions and momentum scalars are held
 * at their values in this run (the loss is piecewise smooth in λ).  No
 * counterpart in the reference, which does not differentiate run_recon.
 * Allocates its checkpoints (niter × Ns images) on first use.  Synchronises
 * `stream`. */
int mslr_pogm_grad(mslr_ctx* ctx, const void* X_true, int32_t niter, double L, double restart_cutoff,
                   double bsig, void* X, double* loss, double* grad_loglam, uint8_t* restarts_host,
                   void* stream);

/* Autotuner (tuned and TF32 forms; no counterpart in the reference).  Times,
 * on the bound context, the launch shapes the library can choose freely —
 * coils per group × frames per chunk of the SENSE normal operator, its lanes
 * (one or two streams) and z-mask CTA variant (two per SM, one per SM, or
 * two per SM of fewer warps), the
 * split-K count of each single-patch scale's Gram, and the eigen stage's CTA
 * variant of each scale with Gram side <= 384 (384 threads, two per SM, or
 * 1024 threads) — and keeps the fastest.  Runs at the end of mslr_bind when
 * the environment has MSLR_AUTOTUNE=1.  The choices change the order of
 * floating-point sums, so results depend on them (to FP32 rounding).  Call
 * before the first POGM step (it uses the POGM buffers as scratch), or the
 * captured iteration is captured again.  mslr_get_tuning writes {coils per
 * group, frames per chunk, split count of scale 0 .. Ns−1 (0: heuristic),
 * lanes, z-mask CTAs per SM, z-mask warps per CTA, eigen CTA threads of
 * scale 0 .. Ns−1}. */
int mslr_autotune(mslr_ctx* ctx, void* stream);
int mslr_get_tuning(const mslr_ctx* ctx, int32_t* values, int32_t cap, int32_t* count);

/* Number of kernels this context has launched so far (host-side count). */
int mslr_launch_count(const mslr_ctx* ctx, uint64_t* count);

/* poweriter_mod (src/mirt_mod.jl:215-238) on the block-diagonal A with
 * x0 = ones: sigma1 = ||A x|| / ||x||, FP64 norms. */
int mslr_power_iter(mslr_ctx* ctx, int32_t niter, double tol, double* sigma1,
                    int32_t* iters_done, void* stream);

/* Measured FP32 FMA throughput of the current device in TFLOP/s (the best of
 * three timed launches of independent FMA chains on every SM), the
 * denominator of the roofline fractions of SIMT-bound kernels.  No
 * counterpart in the reference.  Synchronises `stream`. */
int mslr_fp32_peak(double* tflops, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MSLR_H */
