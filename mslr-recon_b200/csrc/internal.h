// internal.h — context structure and launcher declarations shared by the
// translation units of libmslr.
#pragma once
#include <string>
#include <vector>

#include "common.cuh"

namespace mslr {

// Thread-local error message of the last failing call (context-free calls).
int fail(int code, const std::string& msg);
const std::string& last_error_tls();

// Device-side POGM scalar state (src/mirt_mod.jl:97-184 scalars).  Lives in
// device memory so that one iteration can be captured in a CUDA graph and
// replayed without host round trips.
struct PogmState {
  double told, sig, tnew;
  double alpha, beta, gamma, zeta;
  double restart_cutoff, bsig;
  int iter, niter;
  int flags;               // bit0: sigma-decrease test needed (bsig != 1)
  int pad;
  double red[4];           // last reductions: Σ Re(−g·Δu), ‖g‖², ‖Δu‖², Σ Re(g·gold)
};

// Per-scale SVST workspace layout (all patches of a scale share one layout).
struct SvstWork {
  int n = 0;                 // Gram side
  int64_t np = 0;            // patches
  cf* gram = nullptr;        // np * n * n   Gram, then Householder vectors, then W
  cf* zv = nullptr;          // np * n * n   FP64 tridiagonal eigenvectors, then V (complex64)
  double* aux = nullptr;     // np * n * n   FP64 scratch for the twisted factorisations
  double* vecs = nullptr;    // np * 6 * n   split eigen stage: d, e of T, eigenvalues, √-weights h
  int* rank = nullptr;       // np          number of singular values above β
  cf* split_part = nullptr;  // nsplit * n * n partial Grams (split-K)
  int nsplit = 1;
};

struct Ctx {
  int N[3] = {0, 0, 0};
  int Nc = 0, Nt = 0;
  int64_t K = 0;
  int Ns = 0;
  int form = MSLR_FORM_PLAIN;
  // tuned-form machinery (specialised SENSE kernels, batched SVST, graph): TUNED and TF32
  bool tuned() const { return form == MSLR_FORM_TUNED || form == MSLR_FORM_TF32; }
  // tensor-core mode of the Gram / rebuild products: 0 SIMT FP32, 1 split BF16, 2 TF32
  int tc_mode() const { return form == MSLR_FORM_TF32 ? 2 : form == MSLR_FORM_TUNED ? 1 : 0; }
  int64_t nvox = 0;
  int device = 0;
  std::vector<ScaleGeom> scales;
  std::vector<double> lambdas;   // Ong–Lustig λ_k (scripts/reconstruct.jl:163-169)

  // SENSE
  AxisPlan plan[3];
  cf* d_tw[3] = {nullptr, nullptr, nullptr};     // twiddles exp(-2πik/n)
  cf* d_phase[3] = {nullptr, nullptr, nullptr};  // φ_d(k) = exp(2πi c(k-c)/n)
  cf* d_mod[3] = {nullptr, nullptr, nullptr};    // m_d(j) = exp(2πi j c/n)
  cf* d_smaps_mod = nullptr;   // (Nc, nvox) coil maps × input modulation
  uint32_t* d_mask = nullptr;  // (Nt, nwords) sampling bitmasks
  int nwords = 0;
  int32_t* d_idx = nullptr;    // (Nt, K) 0-based
  cf* d_ahy = nullptr;         // (Nt, nvox) A'y
  double ynorm2 = 0.0;         // ‖y‖² (FP64) of the bound k-space, for dc_cost
  double* d_nuc = nullptr;     // per-patch nuclear norms (cost evaluation)
  int64_t nuc_cap = 0;
  double* d_zero = nullptr;    // device 0.0 (threshold of the values-only eigen mode)
  cf* d_cost_g = nullptr;      // gradient scratch of the cost evaluation (Nt, nvox)
  double* d_cost_part = nullptr;   // FP64 block partials of the cost inner products
  // unrolled-POGM gradient (grad.cu): z_i of every iteration, the adjoint
  // state (x̄, ū, z̄, w, A'A w, scratch image) and the patch-SVST backward
  cf* d_ckpt = nullptr;
  int grad_ckpt_cap = 0;
  cf* d_gbuf = nullptr;
  void* d_vjpw = nullptr;
  size_t vjpw_bytes = 0;
  cf* d_T = nullptr;           // (F, Nc, nvox) per-coil k-space of a chunk of frames
  int F = 1;
  bool bound = false;
  // tuned SENSE kernels (sense_fast.cu): plans and frames per chunk
  bool fast = false;
  alignas(16) unsigned char fplan_raw[3 * 256];   // fast::FPlan x, y, z (fft_fast.cuh)
  int Ffast = 1;
  int nsm = 148;          // SMs of the bound device (persistent grids)
  bool zpre = false;      // z kernels with prefetched slabs fit in shared memory
  bool xypers = false;    // persistent plane kernel with a prefetch buffer fits
  bool spec = false;      // shape-specialised kernels (sense_spec.cu) exist for N
  int spec_xy_ctas = 0;   // resident CTAs of the specialised plane kernel
  int spec_ch = 6;        // coils per group of the specialised normal operator (autotuned)
  int spec_fr = 2;        // frames per chunk (autotuned)
  int spec_zfwd_ctas = 0; // resident CTAs of the specialised forward z kernel
  // four-pass form of the specialised normal operator (default; MSLR_SENSE_PATH=3
  // selects the three-kernel form): resident CTAs of its kernels, and the
  // summed image Σ_k X_k of all frames that its forward plane pass reads
  bool spec_four = true;
  int spec_pfwd_ctas = 0, spec_zmask_ctas = 0, spec_padj_ctas = 0;
  // z-mask kernel variant: 0 two CTAs per SM (64 registers), 1 one CTA per SM
  // (MSLR_ZMASK_CTAS=1), 2 two CTAs per SM with fewer warps (more registers)
  int spec_zmask_var = 0;
  int spec_zmask_ctas_v[3] = {0, 0, 0};   // resident CTAs of each variant
  int spec_zmask_warps[3] = {0, 0, 0};    // warps per CTA of each variant
  // chunks of the four-pass form alternate between two streams ("lanes",
  // each with its own k-space buffer) when spec_lanes == 2 (the default;
  // MSLR_SENSE_LANES=1 keeps one), so one chunk's kernels overlap the other's
  int spec_lanes = 1;
  cudaStream_t sn_stream = nullptr;
  cudaEvent_t sn_fork = nullptr, sn_join = nullptr;
  cf* d_xsum = nullptr;   // (Nt, nvox)
  bool xy_tc = false;     // tensor-core plane pass (DFT products on tcgen05)
  uint32_t* d_dft = nullptr;   // its split-BF16 DFT matrix tiles
  // graph-captured POGM step (tuned form): captured on a private stream the
  // first time pogm_step sees a given X, replayed afterwards
  cudaStream_t gstream = nullptr;
  // concurrent per-scale SVST branches (svst.cu): side streams and fork / join events
  std::vector<cudaStream_t> sv_streams;
  cudaEvent_t sv_fork = nullptr;
  std::vector<cudaEvent_t> sv_join;
  cudaEvent_t gev_in = nullptr, gev_out = nullptr;
  cudaGraphExec_t gexec = nullptr;
  const void* gX = nullptr;
  uint64_t glaunches = 0;
  bool use_graph = true;
  // launch profiling of the specialised normal operator (mslr_normal_op_profile):
  // when on, an event is recorded before and after every kernel of every chunk
  bool prof_on = false;
  std::vector<cudaEvent_t> prof_ev;
  int prof_n = 0;   // events recorded in the current profiled call
  int prof_kernels = 3;   // kernels per chunk of the profiled call (events per chunk: + 1)

  // POGM
  cf* d_U = nullptr;   // (Ns, Nt, nvox)
  cf* d_Z = nullptr;   // (Ns, Nt, nvox) pre-prox iterate z_i
  cf* d_G = nullptr;   // (Nt, nvox) gradient
  cf* d_Gold = nullptr;  // (Nt, nvox) previous gradient (only when bsig != 1)
  cf* d_Y = nullptr;     // (Ns, Nt, nvox) y_i of mom = :pgm / :fpgm (allocated on first use)
  double* d_part = nullptr;   // reduction partials
  int nred_blocks = 0;
  PogmState* d_state = nullptr;
  uint8_t* d_restarts = nullptr;  // niter+1
  int restarts_cap = 0;
  double* d_thr = nullptr;    // device threshold multiplier (ζ for POGM, β for standalone)
  int32_t* d_err = nullptr;   // device error word (kErr* bits), read and cleared by take_error
  int wait_polls = kWaitPolls; // polls of a bounded wait in this context's tcgen05 kernels
  bool pogm_ready = false;

  // SVST
  std::vector<SvstWork> svw;   // one per scale (the plain form shares buffers across scales)
  cf* d_pbuf = nullptr;        // per-patch output buffer for non-partition scales
  size_t pbuf_elems = 0;
  cf* d_img_tmp = nullptr;     // (Nt, nvox) out-of-place staging for in-place calls
  double* d_pthr = nullptr;    // per-patch thresholds (the largest Np of the scales)

  size_t bytes = 0;
  uint64_t launches = 0;   // kernels launched through this context
  std::string err;
};

// ---- device memory helper -------------------------------------------------
int dalloc(Ctx* c, void** p, size_t bytes);
// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) that only ever raises the
// kernel's limit on the current device: the attribute is per process, and a
// context of a smaller shape created later must not lower the limit another
// live context's launches rely on.  Returns the CUDA status.
cudaError_t raise_dyn_smem(const void* func, int bytes);

// ---- device-side errors (api.cu, svst.cu) -----------------------------------
// Error word and wait limit of a context's kernels.
inline DevWait ctx_wait(Ctx* c) {
  DevWait w;
  w.err = c->d_err;
  w.polls = c->wait_polls;
  return w;
}
// Synchronises st, reads and clears the context's error word; returns the
// status its bits map to (MSLR_OK when none is set).
int take_error(Ctx* c, cudaStream_t st);
// Poll count of the bounded waits of the context-free batched SVST calls.
int context_free_polls();
void set_context_free_polls(int polls);

// ---- sense.cu ----------------------------------------------------------------
int sense_setup_tables(Ctx* c);   // twiddles, phases, plans (create time)
int sense_bind(Ctx* c, const cf* smaps, const cf* y, const int32_t* idx, int base,
               cudaStream_t st);
int sense_forward(Ctx* c, const cf* x, cf* y, cudaStream_t st);
int sense_adjoint(Ctx* c, const cf* y, cf* x, cudaStream_t st);
// g = A'(A Σ_k X_k − y) (subtract) or A'A Σ_k X_k
int normal_op(Ctx* c, const cf* X, int ns, int64_t sstride, cf* g, bool subtract,
              cudaStream_t st);

// ---- sense_fast.cu (tuned form) ------------------------------------------------
bool sense_fast_setup(Ctx* c);
int normal_op_fast(Ctx* c, const cf* X, int ns, int64_t sstride, cf* g, bool subtract,
                   cudaStream_t st);
int sense_forward_fast(Ctx* c, const cf* x, cf* y, cudaStream_t st);
int sense_adjoint_fast(Ctx* c, const cf* y, cf* x, cudaStream_t st);

// ---- sense_spec.cu (tuned form, compiled shapes) ---------------------------------
bool sense_spec_setup(Ctx* c);
int normal_op_spec(Ctx* c, const cf* X, int ns, int64_t sstride, cf* g, bool subtract,
                   cudaStream_t st);

// ---- svst.cu -----------------------------------------------------------------
int svst_setup(Ctx* c);   // workspaces (create time)
// img_out = patchSVST(img_in) for scale s with threshold (*thr_dev) * lam
int patch_svst_all(Ctx* c, const double* thr_dev, const cf* Zin, cf* Xout, cudaStream_t st);
int patch_svst(Ctx* c, int s, const double* thr_dev, double lam, const cf* img_in, cf* img_out,
               cudaStream_t st, int thr_per_patch = 0);
// per-patch thresholds of a scale (patchSVST(img, λs, ...), src/recon.jl:263-268)
int patch_svst_lambdas(Ctx* c, int s, const double* lambdas_host, const cf* img_in, cf* img_out,
                       cudaStream_t st);
// nuclear norms of every patch of scale s of img, in patch order (synchronises st)
int patch_nucnorms(Ctx* c, int s, const cf* img, std::vector<double>& out, cudaStream_t st);
int geom_build(const int N[3], int Nt, const int ps_in[3], const int ss_in[3], ScaleGeom* g);
int geom_upload(ScaleGeom* g, const int N[3]);
void geom_free(ScaleGeom* g);

// ---- eig.cu --------------------------------------------------------------------
// One group of patches that share a Gram side n and a threshold multiplier.
struct EigSegment {
  int n;
  int64_t np;
  cf* gram;      // np × n × n: Gram in (lower triangle read), Householder vectors out
  cf* zv;        // np × n × n: Ṽ = V diag(√h) out, conjugated, row-major (W = Ṽ Ṽᴴ)
  double* aux;   // np × n × n scratch
  int* rank;     // np
  double lam;
  int big = 0;             // 1: the 1024-thread CTA variant even when n <= 384
  double* nuc = nullptr;   // when set: per-patch Σ √λ above the threshold only (no vectors, no W)
  double* lam_out = nullptr;   // when set: every eigenpair — V (row-major, G = V Λ Vᴴ) in zv
                               // and the eigenvalues (descending, np × n) here; threshold unused
  double* side = nullptr;      // np × 6n FP64 scratch; when set (and 64 <= n <= 384), the stage
                               // runs as three launches (tridiagonalise, eigenpairs of T, V = Q Z)
};
// Adds the number of kernels launched to *launches when given.
int eig_launch_multi(int nseg, const EigSegment* segs, const double* thr, int thr_per_patch,
                     cudaStream_t st, uint64_t* launches = nullptr);
int eig2_prepare(int nmax);
int eig2_launch(int n, int64_t np, cf* gram, cf* zv, float* aux, int* rank, const double* thr,
                int thr_per_patch, double lam, cudaStream_t st, int big = 0, double* side = nullptr,
                uint64_t* launches = nullptr);

// ---- cost evaluation (svst.cu, cost.cu) ------------------------------------------
int patch_nucnorm_all(Ctx* c, const cf* X, double* reg_out, cudaStream_t st);
int data_norm2(Ctx* c, const cf* y, double* out, cudaStream_t st);
int dc_cost_eval(Ctx* c, const cf* X, int ns, double* dc_out, cudaStream_t st);

// ---- pogm.cu -----------------------------------------------------------------
int pogm_setup(Ctx* c);
int pogm_begin(Ctx* c, cf* X, int niter, double L, double cutoff, double bsig, cudaStream_t st);
int pogm_step(Ctx* c, cf* X, cudaStream_t st);
// sharded iteration (sharded.py): the rank-local half, the decision from the
// totals over the ranks, the current scalars
int pogm_step_local(Ctx* c, cf* X, cf* Zout, double* sums_dev, cudaStream_t st);
int pogm_step_decide(Ctx* c, const double* sums_dev, cudaStream_t st);
int pogm_run_options(Ctx* c, cf* X, int niter, double L, double mu, int mom, int restart,
                     double cutoff, double bsig, uint8_t* restarts_h, cudaStream_t st);
int pogm_scalars(Ctx* c, double* out, cudaStream_t st);
int patch_gram_out(Ctx* c, int s, const cf* img, cf* gram_out, cudaStream_t st);
int patch_svst_from_gram(Ctx* c, int s, double beta, const cf* gram, const cf* img_in, cf* img_out,
                         cudaStream_t st);
int init_x0(Ctx* c, cf* X, cudaStream_t st);
int power_iter(Ctx* c, int niter, double tol, double* sigma1, int* iters, cudaStream_t st);
int set_scalar(double* dst, double v, cudaStream_t st);

// ---- autotuner (api.cu; sense_spec.cu, svst.cu) ---------------------------------
int tune_sense_chunks(Ctx* c, cudaStream_t st);
int tune_svst_splits(Ctx* c, cudaStream_t st);
int tune_sense_variants(Ctx* c, cudaStream_t st);
int tune_eig_variants(Ctx* c, cudaStream_t st);
int autotune(Ctx* c, cudaStream_t st);
// milliseconds per call of fn(), timed with events on st after one warm-up call
template <class Fn>
int time_ms(cudaStream_t st, int reps, float* ms, Fn&& fn) {
  int rc = fn();
  if (rc) return rc;
  cudaEvent_t e0, e1;
  MSLR_CUDA_TRY(cudaEventCreate(&e0));
  MSLR_CUDA_TRY(cudaEventCreate(&e1));
  cudaEventRecord(e0, st);
  for (int i = 0; i < reps && !rc; ++i) rc = fn();
  cudaEventRecord(e1, st);
  const cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(MSLR_ERR_CUDA, cudaGetErrorString(e));
  *ms = t / reps;
  return MSLR_OK;
}

// ---- set-up of run_recon's inputs (setup.cu) ---------------------------------
int sos_normalize(const int N[3], int Nc, const cf* in, cf* out, cudaStream_t st);
int sampling(const int N[3], int Nc, int Nt, const cf* ksp, int64_t* K, int32_t* idx, cf* y,
             int64_t K_cap, cudaStream_t st);
int prepare_scale(Ctx* c, const cf* smaps, cf* y, const int32_t* idx, double* scale_out, cudaStream_t st);

// ---- unrolled-POGM gradient (grad.cu; patch-SVST backward in svst.cu) ---------
struct PatchMap;
int set_lambdas(Ctx* c, const double* lam);
int pogm_grad(Ctx* c, const cf* Xtrue, int niter, double L, double cutoff, double bsig, cf* X,
              double* loss, double* grad, uint8_t* restarts_h, cudaStream_t st);
int svst_vjp_setup(Ctx* c);
int svst_vjp_scale(Ctx* c, int s, const cf* z, const cf* xbar, double beta, cf* zbar, cf* tmp,
                   double* bbar, cudaStream_t st);
int xgram_launch(const cf* imgO, const cf* imgM, const PatchMap& m, int64_t np, cf* out, cf* part,
                 int nsplit, cudaStream_t st);
int bgemm_launch(int opa, int opb, const cf* A, const cf* B, cf* C, int n, int64_t np, cudaStream_t st);
int divdiff_launch(const cf* D, const double* lam, const cf* V, double beta, int n, int64_t np, cf* E,
                   cf* T3, double* bbar, cudaStream_t st);
int vjp_rebuild_launch(const cf* xb, const cf* z, const cf* W, const cf* K, const PatchMap& m,
                       int64_t np, cf* out, int direct, cudaStream_t st);
int div_count_launch(const cf* img, const PatchMap& m, const int* cover, cf* out, cudaStream_t st);
int patch_sum_launch(const cf* P, const PatchMap& m, const int* cover, cf* img, cudaStream_t st);

}  // namespace mslr
