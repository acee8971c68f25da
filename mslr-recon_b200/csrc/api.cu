// api.cu — the extern "C" entry points declared in include/mslr.h.
#include <cmath>
#include <cstring>

#include <string>

#include <cstdlib>
#include <map>
#include <mutex>
#include <vector>
#include "internal.h"
#include "patchmap.cuh"

struct mslr_ctx : public mslr::Ctx {};

namespace mslr {

static thread_local std::string tls_err;

int fail(int code, const std::string& msg) {
  tls_err = msg;
  return code;
}
const std::string& last_error_tls() { return tls_err; }

int dalloc(Ctx* c, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(MSLR_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " +
                                    cudaGetErrorString(e));
  }
  c->bytes += bytes;
  return MSLR_OK;
}

cudaError_t raise_dyn_smem(const void* func, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> cur;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  int& have = cur[{dev, func}];
  if (bytes <= have) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}

// defined in svst.cu
int patches_op(const int N[3], int Nt, const int ps[3], const int ss[3], const cf* src, cf* dst,
               bool to_patches, cudaStream_t st);
size_t svst_batch_bytes(int mrows, int ncols, int batch);
int svst_batch(int mrows, int ncols, int batch, const double* betas, const cf* in, cf* out,
               void* ws, size_t ws_bytes, int form, cudaStream_t st);
int svst_batch_noalloc(int mrows, int ncols, int batch, const double* betas, const cf* in, cf* out,
                       cudaStream_t st);

static void free_ctx(mslr_ctx* c) {
  void* ptrs[] = {c->d_tw[0], c->d_tw[1], c->d_tw[2], c->d_phase[0], c->d_phase[1], c->d_phase[2],
                  c->d_mod[0], c->d_mod[1], c->d_mod[2], c->d_smaps_mod, c->d_mask, c->d_idx,
                  c->d_ahy, c->d_T, c->d_U, c->d_Z, c->d_G, c->d_Gold, c->d_Y, c->d_part, c->d_state,
                  c->d_restarts, c->d_thr, c->d_err, c->d_pbuf, c->d_img_tmp};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (auto& w : c->svw)
    if (w.gram) cudaFree(w.gram);
  for (auto& g : c->scales) geom_free(&g);
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->gev_in) cudaEventDestroy(c->gev_in);
  if (c->gev_out) cudaEventDestroy(c->gev_out);
  if (c->gstream) cudaStreamDestroy(c->gstream);
  for (cudaStream_t x : c->sv_streams) cudaStreamDestroy(x);
  for (cudaEvent_t e : c->sv_join) cudaEventDestroy(e);
  if (c->sv_fork) cudaEventDestroy(c->sv_fork);
  if (c->d_nuc) cudaFree(c->d_nuc);
  if (c->d_dft) cudaFree(c->d_dft);
  if (c->d_zero) cudaFree(c->d_zero);
  if (c->d_cost_g) cudaFree(c->d_cost_g);
  if (c->d_cost_part) cudaFree(c->d_cost_part);
  if (c->d_ckpt) cudaFree(c->d_ckpt);
  if (c->d_gbuf) cudaFree(c->d_gbuf);
  if (c->d_vjpw) cudaFree(c->d_vjpw);
  if (c->d_xsum) cudaFree(c->d_xsum);
  if (c->d_pthr) cudaFree(c->d_pthr);
  if (c->sn_stream) cudaStreamDestroy(c->sn_stream);
  if (c->sn_fork) cudaEventDestroy(c->sn_fork);
  if (c->sn_join) cudaEventDestroy(c->sn_join);
  delete c;
}

static int ctx_fail(Ctx* c, int code) {
  if (c) c->err = tls_err;
  return code;
}

int take_error(Ctx* c, cudaStream_t st) {
  int32_t herr = 0;
  cudaError_t e = cudaMemcpyAsync(&herr, c->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(MSLR_ERR_CUDA, cudaGetErrorString(e));
  if (!herr) return MSLR_OK;
  e = cudaMemsetAsync(c->d_err, 0, sizeof(int32_t), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(MSLR_ERR_CUDA, cudaGetErrorString(e));
  if (herr & kErrNonfinite) return fail(MSLR_ERR_NONFINITE, "non-finite value in the POGM restart sums");
  if (herr & kErrMmaWait)
    return fail(MSLR_ERR_CUDA, "a tensor-core kernel's bounded wait for its MMAs timed out; "
                               "results since the last check are not valid");
  if (herr & kErrBulkWait)
    return fail(MSLR_ERR_CUDA, "a SENSE kernel's bounded wait for a bulk copy timed out; "
                               "results since the last check are not valid");
  return fail(MSLR_ERR_CUDA, "device error word " + std::to_string(herr));
}

}  // namespace mslr

using namespace mslr;

#define CTX_CHECK(ctx)                                                  \
  do {                                                                  \
    if (!(ctx)) return fail(MSLR_ERR_ARG, "null context");              \
  } while (0)
#define CTX_RET(ctx, expr)                                              \
  do {                                                                  \
    int _rc = (expr);                                                   \
    if (_rc) return ctx_fail((ctx), _rc);         \
  } while (0)

extern "C" {

int mslr_abi_version(void) { return MSLR_ABI_VERSION; }

const char* mslr_last_error(const mslr_ctx* ctx) {
  if (ctx) return ctx->err.c_str();
  return tls_err.c_str();
}

int mslr_patch_geometry(const int32_t N[3], const int32_t patch[3], const int32_t stride[3],
                        int32_t ps_out[3], int32_t nsteps_out[3], int64_t* Np_out,
                        int32_t* starts) {
  if (!N || !patch || !stride) return fail(MSLR_ERR_ARG, "null argument");
  for (int d = 0; d < 3; ++d)
    if (N[d] <= 0) return fail(MSLR_ERR_ARG, "image dimensions must be positive");
  ScaleGeom g;
  const int n3[3] = {N[0], N[1], N[2]};
  const int p3[3] = {patch[0], patch[1], patch[2]};
  const int s3[3] = {stride[0], stride[1], stride[2]};
  int rc = geom_build(n3, 1, p3, s3, &g);
  if (rc) return rc;
  for (int d = 0; d < 3; ++d) {
    if (ps_out) ps_out[d] = g.ps[d];
    if (nsteps_out) nsteps_out[d] = g.nsteps[d];
  }
  if (Np_out) *Np_out = g.Np;
  if (starts)
    for (size_t i = 0; i < g.h_starts.size(); ++i) starts[i] = g.h_starts[i];
  return MSLR_OK;
}

int mslr_img2patches(const int32_t N[3], int32_t Nt, const int32_t patch[3],
                     const int32_t stride[3], const void* img, void* P, void* stream) {
  if (!N || !patch || !stride || !img || !P || Nt <= 0) return fail(MSLR_ERR_ARG, "bad argument");
  const int n3[3] = {N[0], N[1], N[2]}, p3[3] = {patch[0], patch[1], patch[2]},
            s3[3] = {stride[0], stride[1], stride[2]};
  return patches_op(n3, Nt, p3, s3, reinterpret_cast<const cf*>(img), reinterpret_cast<cf*>(P),
                    true, reinterpret_cast<cudaStream_t>(stream));
}

int mslr_patches2img(const int32_t N[3], int32_t Nt, const int32_t patch[3],
                     const int32_t stride[3], const void* P, void* img, void* stream) {
  if (!N || !patch || !stride || !img || !P || Nt <= 0) return fail(MSLR_ERR_ARG, "bad argument");
  const int n3[3] = {N[0], N[1], N[2]}, p3[3] = {patch[0], patch[1], patch[2]},
            s3[3] = {stride[0], stride[1], stride[2]};
  return patches_op(n3, Nt, p3, s3, reinterpret_cast<const cf*>(P), reinterpret_cast<cf*>(img),
                    false, reinterpret_cast<cudaStream_t>(stream));
}

int mslr_svst_batch_workspace(int32_t m, int32_t n, int32_t batch, size_t* bytes) {
  if (m <= 0 || n <= 0 || batch <= 0 || !bytes) return fail(MSLR_ERR_ARG, "bad argument");
  if (std::min(m, n) > 1024) return fail(MSLR_ERR_UNSUPPORTED, "min(m, n) must be <= 1024");
  *bytes = svst_batch_bytes(m, n, batch);
  return MSLR_OK;
}

int mslr_svst_batch(int32_t m, int32_t n, int32_t batch, const double* betas, const void* in,
                    void* out, void* workspace, size_t workspace_bytes, int32_t form,
                    void* stream) {
  if (m <= 0 || n <= 0 || batch <= 0 || !betas || !in || !out || !workspace)
    return fail(MSLR_ERR_ARG, "bad argument");
  if (std::min(m, n) > 1024) return fail(MSLR_ERR_UNSUPPORTED, "min(m, n) must be <= 1024");
  for (int b = 0; b < batch; ++b)
    if (!(betas[b] >= 0.0) || !std::isfinite(betas[b]))
      return fail(MSLR_ERR_ARG, "thresholds must be finite and non-negative");
  if (form != MSLR_FORM_PLAIN && form != MSLR_FORM_TUNED && form != MSLR_FORM_TF32)
    return fail(MSLR_ERR_ARG, "unknown form");
  return svst_batch(m, n, batch, betas, reinterpret_cast<const cf*>(in), reinterpret_cast<cf*>(out),
                    workspace, workspace_bytes, form, reinterpret_cast<cudaStream_t>(stream));
}

int mslr_svst_batch_noalloc(int32_t m, int32_t n, int32_t batch, const double* betas,
                            const void* in, void* out, void* stream) {
  if (m <= 0 || n <= 0 || batch <= 0 || !betas || !in || !out)
    return fail(MSLR_ERR_ARG, "bad argument");
  if (std::min(m, n) > 1024) return fail(MSLR_ERR_UNSUPPORTED, "min(m, n) must be <= 1024");
  for (int b = 0; b < batch; ++b)
    if (!(betas[b] >= 0.0) || !std::isfinite(betas[b]))
      return fail(MSLR_ERR_ARG, "thresholds must be finite and non-negative");
  return svst_batch_noalloc(m, n, batch, betas, reinterpret_cast<const cf*>(in),
                            reinterpret_cast<cf*>(out), reinterpret_cast<cudaStream_t>(stream));
}

int mslr_create(const int32_t N[3], int32_t Nc, int32_t Nt, int64_t K, int32_t n_scales,
                const int32_t* patch, const int32_t* stride, int32_t form, mslr_ctx** out) {
  if (!out) return fail(MSLR_ERR_ARG, "null output pointer");
  *out = nullptr;
  if (!N || !patch || !stride) return fail(MSLR_ERR_ARG, "null argument");
  if (N[0] <= 0 || N[1] <= 0 || N[2] <= 0 || Nc <= 0 || Nt <= 0 || K <= 0 || n_scales <= 0)
    return fail(MSLR_ERR_ARG, "dimensions, coils, frames, samples and scales must be positive");
  if (form != MSLR_FORM_PLAIN && form != MSLR_FORM_TUNED && form != MSLR_FORM_TF32)
    return fail(MSLR_ERR_ARG, "unknown form");
  const int64_t nvox = (int64_t)N[0] * N[1] * N[2];
  if (K > nvox) return fail(MSLR_ERR_ARG, "more samples per frame than k-space points");
  mslr_ctx* c = new mslr_ctx();
  c->N[0] = N[0];
  c->N[1] = N[1];
  c->N[2] = N[2];
  c->Nc = Nc;
  c->Nt = Nt;
  c->K = K;
  c->Ns = n_scales;
  c->form = form;
  c->nvox = nvox;
  cudaGetDevice(&c->device);
  int rc = MSLR_OK;
  c->scales.resize(n_scales);
  for (int k = 0; k < n_scales && !rc; ++k) {
    const int p3[3] = {patch[3 * k], patch[3 * k + 1], patch[3 * k + 2]};
    const int s3[3] = {stride[3 * k], stride[3 * k + 1], stride[3 * k + 2]};
    rc = geom_build(c->N, Nt, p3, s3, &c->scales[k]);
    if (!rc && c->scales[k].n > 1024)
      rc = fail(MSLR_ERR_UNSUPPORTED, "min(patch voxels, Nt) must be <= 1024");
    if (!rc) rc = geom_upload(&c->scales[k], c->N);
    // Ong–Lustig λ with the unclamped patch size (scripts/reconstruct.jl:163-169)
    const double pk = (double)p3[0] * p3[1] * p3[2];
    c->lambdas.push_back(std::sqrt(pk) + std::sqrt((double)Nt) +
                         std::sqrt(std::log((double)nvox * Nt / std::max(pk, (double)Nt))));
  }
  if (!rc) rc = dalloc(c, (void**)&c->d_thr, 64 * sizeof(double));
  if (!rc) rc = dalloc(c, (void**)&c->d_err, 64);
  if (!rc) rc = sense_setup_tables(c);
  if (!rc) rc = pogm_setup(c);
  if (!rc) rc = svst_setup(c);
  if (rc) {
    free_ctx(c);
    return rc;
  }
  *out = c;
  return MSLR_OK;
}

int mslr_destroy(mslr_ctx* ctx) {
  if (!ctx) return MSLR_OK;
  cudaDeviceSynchronize();
  free_ctx(ctx);
  return MSLR_OK;
}

int mslr_workspace_bytes(const mslr_ctx* ctx, size_t* bytes) {
  CTX_CHECK(ctx);
  if (!bytes) return fail(MSLR_ERR_ARG, "null output pointer");
  *bytes = ctx->bytes;
  return MSLR_OK;
}

int mslr_bind(mslr_ctx* ctx, const void* smaps, const void* y, const int32_t* idx,
              int32_t index_base, void* stream) {
  CTX_CHECK(ctx);
  if (!smaps || !y || !idx) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  if (index_base != 0 && index_base != 1)
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "index_base must be 0 or 1"));
  CTX_RET(ctx, sense_bind(ctx, reinterpret_cast<const cf*>(smaps), reinterpret_cast<const cf*>(y),
                          idx, index_base, reinterpret_cast<cudaStream_t>(stream)));
  const char* at = std::getenv("MSLR_AUTOTUNE");
  if (at && std::string(at) == "1" && ctx->tuned())
    CTX_RET(ctx, autotune(ctx, reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

#define NEED_BOUND(ctx)                                                                   \
  do {                                                                                    \
    if (!(ctx)->bound) return ctx_fail(ctx, fail(MSLR_ERR_STATE, "mslr_bind not called")); \
  } while (0)

int mslr_sense_forward(mslr_ctx* ctx, const void* x, void* y, void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!x || !y) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, sense_forward(ctx, reinterpret_cast<const cf*>(x), reinterpret_cast<cf*>(y),
                             reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_sense_adjoint(mslr_ctx* ctx, const void* y, void* x, void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!x || !y) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, sense_adjoint(ctx, reinterpret_cast<const cf*>(y), reinterpret_cast<cf*>(x),
                             reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_normal_op(mslr_ctx* ctx, const void* X, int32_t ns_in, void* g, int32_t subtract_data,
                   void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!X || !g || ns_in <= 0) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad argument"));
  CTX_RET(ctx, normal_op(ctx, reinterpret_cast<const cf*>(X), ns_in, (int64_t)ctx->Nt * ctx->nvox,
                         reinterpret_cast<cf*>(g), subtract_data != 0,
                         reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_normal_op_profile(mslr_ctx* ctx, const void* X, int32_t ns_in, void* g, void* stream,
                           double* kernel_ms, int64_t* launches_per_kernel) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!X || !g || ns_in <= 0 || !kernel_ms || !launches_per_kernel)
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad argument"));
  if (!ctx->spec)
    return ctx_fail(ctx, fail(MSLR_ERR_UNSUPPORTED,
                              "launch profiling needs the shape-specialised SENSE kernels"));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  ctx->prof_on = true;
  ctx->prof_n = 0;
  const int rc = normal_op(ctx, reinterpret_cast<const cf*>(X), ns_in, (int64_t)ctx->Nt * ctx->nvox,
                           reinterpret_cast<cf*>(g), true, st);
  ctx->prof_on = false;
  if (rc) return ctx_fail(ctx, rc);
  const int nk = ctx->prof_kernels, per = nk + 1;
  if (ctx->prof_n == 0 || ctx->prof_n % per)
    return ctx_fail(ctx, fail(MSLR_ERR_CUDA, "profiling events out of step"));
  cudaError_t e = cudaEventSynchronize(ctx->prof_ev[ctx->prof_n - 1]);
  if (e != cudaSuccess) return ctx_fail(ctx, fail(MSLR_ERR_CUDA, cudaGetErrorString(e)));
  double tot[4] = {0.0, 0.0, 0.0, 0.0};
  const int chunks = ctx->prof_n / per;
  for (int q = 0; q < chunks; ++q)
    for (int k = 0; k < nk; ++k) {
      float ms = 0.f;
      e = cudaEventElapsedTime(&ms, ctx->prof_ev[per * q + k], ctx->prof_ev[per * q + k + 1]);
      if (e != cudaSuccess) return ctx_fail(ctx, fail(MSLR_ERR_CUDA, cudaGetErrorString(e)));
      tot[k] += ms;
    }
  for (int k = 0; k < 4; ++k) {
    kernel_ms[k] = (k < nk && chunks) ? tot[k] / chunks : 0.0;
    launches_per_kernel[k] = k < nk ? chunks : 0;
  }
  CTX_RET(ctx, take_error(ctx, st));
  return MSLR_OK;
}

int mslr_patch_svst(mslr_ctx* ctx, int32_t scale, double beta, const void* img_in, void* img_out,
                    void* stream) {
  CTX_CHECK(ctx);
  if (scale < 0 || scale >= ctx->Ns || !img_in || !img_out)
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad argument"));
  if (!(beta >= 0.0) || !std::isfinite(beta))
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "beta must be finite and non-negative"));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  CTX_RET(ctx, set_scalar(ctx->d_thr + 1, beta, st));
  CTX_RET(ctx, patch_svst(ctx, scale, ctx->d_thr + 1, 1.0, reinterpret_cast<const cf*>(img_in),
                          reinterpret_cast<cf*>(img_out), st));
  return MSLR_OK;
}

int mslr_patch_svst_lambdas(mslr_ctx* ctx, int32_t scale, const double* lambdas, const void* img_in,
                            void* img_out, void* stream) {
  CTX_CHECK(ctx);
  if (scale < 0 || scale >= ctx->Ns || !lambdas || !img_in || !img_out)
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad argument"));
  for (int64_t ip = 0; ip < ctx->scales[scale].Np; ++ip)
    if (!(lambdas[ip] >= 0.0) || !std::isfinite(lambdas[ip]))
      return ctx_fail(ctx, fail(MSLR_ERR_ARG, "thresholds must be finite and non-negative"));
  CTX_RET(ctx, patch_svst_lambdas(ctx, scale, lambdas, reinterpret_cast<const cf*>(img_in),
                                  reinterpret_cast<cf*>(img_out), reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_patch_nucnorm(mslr_ctx* ctx, int32_t scale, const double* lambdas, const void* img, double* cost,
                       void* stream) {
  CTX_CHECK(ctx);
  if (scale < 0 || scale >= ctx->Ns || !img || !cost) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad argument"));
  std::vector<double> h;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  CTX_RET(ctx, patch_nucnorms(ctx, scale, reinterpret_cast<const cf*>(img), h, st));
  CTX_RET(ctx, take_error(ctx, st));
  double tot = 0.0;
  if (lambdas) {   // Σ_ip λ_ip Σσ_ip / Np (src/recon.jl:154-166)
    for (size_t ip = 0; ip < h.size(); ++ip) tot += h[ip] > 0.0 ? lambdas[ip] * h[ip] : 0.0;
    tot /= (double)h.size();
  } else {         // Σ_ip Σσ_ip (src/recon.jl:138-146)
    for (double v : h) tot += v;
  }
  *cost = tot;
  return MSLR_OK;
}

int mslr_init_x0(mslr_ctx* ctx, void* X, void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!X) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, init_x0(ctx, reinterpret_cast<cf*>(X), reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

static int check_pogm_args(mslr_ctx* ctx, int32_t niter, double L, double cutoff, double bsig) {
  // src/mirt_mod.jl:88-93
  if (niter < 0) return fail(MSLR_ERR_ARG, "niter must be >= 0");
  if (!(L > 0.0) || !std::isfinite(L)) return fail(MSLR_ERR_ARG, "f_L must be positive and finite");
  if (!(bsig >= 0.0)) return fail(MSLR_ERR_ARG, "bsig < 0");
  if (!(std::fabs(cutoff) < 1.0)) return fail(MSLR_ERR_ARG, "restart_cutoff must satisfy |c| < 1");
  (void)ctx;
  return MSLR_OK;
}

int mslr_pogm_begin(mslr_ctx* ctx, void* X, int32_t niter, double L, double restart_cutoff,
                    double bsig, void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!X) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, check_pogm_args(ctx, niter, L, restart_cutoff, bsig));
  CTX_RET(ctx, pogm_begin(ctx, reinterpret_cast<cf*>(X), niter, L, restart_cutoff, bsig,
                          reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_pogm_step(mslr_ctx* ctx, void* X, void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!ctx->pogm_ready) return ctx_fail(ctx, fail(MSLR_ERR_STATE, "mslr_pogm_begin not called"));
  if (!X) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, pogm_step(ctx, reinterpret_cast<cf*>(X), reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_pogm_restarts(mslr_ctx* ctx, uint8_t* restarts_host, void* stream) {
  CTX_CHECK(ctx);
  if (!ctx->pogm_ready || !ctx->d_restarts)
    return ctx_fail(ctx, fail(MSLR_ERR_STATE, "mslr_pogm_begin not called"));
  if (!restarts_host) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(restarts_host, ctx->d_restarts, ctx->restarts_cap,
                                  cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return ctx_fail(ctx, fail(MSLR_ERR_CUDA, cudaGetErrorString(e)));
  CTX_RET(ctx, take_error(ctx, st));
  return MSLR_OK;
}

int mslr_pogm_run(mslr_ctx* ctx, void* X, int32_t niter, double L, double restart_cutoff,
                  double bsig, uint8_t* restarts_host, void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!X) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, check_pogm_args(ctx, niter, L, restart_cutoff, bsig));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  CTX_RET(ctx, pogm_begin(ctx, reinterpret_cast<cf*>(X), niter, L, restart_cutoff, bsig, st));
  for (int i = 0; i < niter; ++i)
    CTX_RET(ctx, pogm_step(ctx, reinterpret_cast<cf*>(X), st));
  if (restarts_host) {
    cudaError_t e = cudaMemcpyAsync(restarts_host, ctx->d_restarts, (size_t)niter + 1,
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx_fail(ctx, fail(MSLR_ERR_CUDA, cudaGetErrorString(e)));
  }
  CTX_RET(ctx, take_error(ctx, st));
  return MSLR_OK;
}

int mslr_pogm_run_costs(mslr_ctx* ctx, void* X, int32_t niter, double L, double restart_cutoff,
                        double bsig, uint8_t* restarts_host, double* dc_costs_host,
                        double* reg_costs_host, void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!X) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, check_pogm_args(ctx, niter, L, restart_cutoff, bsig));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cf* Xc = reinterpret_cast<cf*>(X);
  // the logger's costs at X0 and after every iteration (scripts/reconstruct.jl:204-205)
  auto log_costs = [&](int it) -> int {
    if (dc_costs_host)
      if (int rc = dc_cost_eval(ctx, Xc, ctx->Ns, &dc_costs_host[it], st)) return rc;
    if (reg_costs_host)
      if (int rc = patch_nucnorm_all(ctx, Xc, &reg_costs_host[it], st)) return rc;
    return MSLR_OK;
  };
  CTX_RET(ctx, pogm_begin(ctx, Xc, niter, L, restart_cutoff, bsig, st));
  CTX_RET(ctx, log_costs(0));
  for (int i = 0; i < niter; ++i) {
    CTX_RET(ctx, pogm_step(ctx, Xc, st));
    CTX_RET(ctx, log_costs(i + 1));
  }
  if (restarts_host) {
    cudaError_t e = cudaMemcpyAsync(restarts_host, ctx->d_restarts, (size_t)niter + 1,
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx_fail(ctx, fail(MSLR_ERR_CUDA, cudaGetErrorString(e)));
  }
  CTX_RET(ctx, take_error(ctx, st));
  return MSLR_OK;
}

int mslr_pogm_run_options(mslr_ctx* ctx, void* X, int32_t niter, double L, double mu, int32_t mom,
                          int32_t restart, double restart_cutoff, double bsig, uint8_t* restarts_host,
                          void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!X) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, check_pogm_args(ctx, niter, L, restart_cutoff, bsig));
  // src/mirt_mod.jl:88-93
  if (mom < MSLR_MOM_PGM || mom > MSLR_MOM_POGM) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad mom"));
  if (restart < MSLR_RESTART_NONE || restart > MSLR_RESTART_FR)
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad restart"));
  if (!(mu >= 0.0)) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "f_mu < 0"));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (mom == MSLR_MOM_POGM && restart == MSLR_RESTART_GR && mu == 0.0) {
    // run_recon's own choice: the fused, graph-replayed iteration
    ctx->err.clear();
    return mslr_pogm_run(ctx, X, niter, L, restart_cutoff, bsig, restarts_host, stream);
  }
  CTX_RET(ctx, pogm_run_options(ctx, reinterpret_cast<cf*>(X), niter, L, mu, mom, restart,
                                restart_cutoff, bsig, restarts_host, st));
  CTX_RET(ctx, take_error(ctx, st));
  return MSLR_OK;
}

int mslr_pogm_step_local(mslr_ctx* ctx, void* X, void* Z, double* sums_dev, void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!ctx->pogm_ready) return ctx_fail(ctx, fail(MSLR_ERR_STATE, "mslr_pogm_begin not called"));
  if (!X || !Z || !sums_dev) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, pogm_step_local(ctx, reinterpret_cast<cf*>(X), reinterpret_cast<cf*>(Z), sums_dev,
                               reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_pogm_step_decide(mslr_ctx* ctx, const double* sums_dev, void* stream) {
  CTX_CHECK(ctx);
  if (!ctx->pogm_ready) return ctx_fail(ctx, fail(MSLR_ERR_STATE, "mslr_pogm_begin not called"));
  if (!sums_dev) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, pogm_step_decide(ctx, sums_dev, reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_pogm_scalars(mslr_ctx* ctx, double* alpha_beta_gamma_zeta, void* stream) {
  CTX_CHECK(ctx);
  if (!ctx->pogm_ready) return ctx_fail(ctx, fail(MSLR_ERR_STATE, "mslr_pogm_begin not called"));
  if (!alpha_beta_gamma_zeta) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, pogm_scalars(ctx, alpha_beta_gamma_zeta, reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_patch_gram(mslr_ctx* ctx, int32_t scale, const void* img, void* gram, void* stream) {
  CTX_CHECK(ctx);
  if (scale < 0 || scale >= ctx->Ns || !img || !gram) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad argument"));
  CTX_RET(ctx, patch_gram_out(ctx, scale, reinterpret_cast<const cf*>(img), reinterpret_cast<cf*>(gram),
                              reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_patch_svst_gram(mslr_ctx* ctx, int32_t scale, double beta, const void* gram, const void* img_in,
                         void* img_out, void* stream) {
  CTX_CHECK(ctx);
  if (scale < 0 || scale >= ctx->Ns || !gram || !img_in || !img_out)
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad argument"));
  if (!(beta >= 0.0) || !std::isfinite(beta))
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "beta must be finite and non-negative"));
  CTX_RET(ctx, patch_svst_from_gram(ctx, scale, beta, reinterpret_cast<const cf*>(gram),
                                    reinterpret_cast<const cf*>(img_in), reinterpret_cast<cf*>(img_out),
                                    reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_autotune(mslr_ctx* ctx, void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!ctx->tuned()) return MSLR_OK;
  CTX_RET(ctx, autotune(ctx, reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_get_tuning(const mslr_ctx* ctx, int32_t* values, int32_t cap, int32_t* count) {
  CTX_CHECK(ctx);
  if (!count || (cap > 0 && !values)) return fail(MSLR_ERR_ARG, "null argument");
  std::vector<int32_t> v = {ctx->spec_ch, ctx->spec_fr};
  for (const auto& g : ctx->scales) v.push_back(g.nsplit_tuned > 0 ? g.nsplit_tuned : 0);
  v.push_back(ctx->spec_lanes);
  v.push_back(ctx->spec_zmask_var == 1 ? 1 : 2);
  v.push_back(ctx->spec_zmask_warps[ctx->spec_zmask_var]);
  for (const auto& g : ctx->scales) v.push_back(g.n > 384 || g.eig_big ? 1024 : 384);
  *count = (int32_t)v.size();
  for (int32_t i = 0; i < cap && i < (int32_t)v.size(); ++i) values[i] = v[i];
  return MSLR_OK;
}

int mslr_sos_normalize(const int32_t N[3], int32_t Nc, const void* smaps_raw, void* smaps_out,
                       void* stream) {
  if (!N || !smaps_raw || !smaps_out || Nc <= 0 || N[0] <= 0 || N[1] <= 0 || N[2] <= 0)
    return fail(MSLR_ERR_ARG, "bad argument");
  const int n3[3] = {N[0], N[1], N[2]};
  return sos_normalize(n3, Nc, reinterpret_cast<const cf*>(smaps_raw), reinterpret_cast<cf*>(smaps_out),
                       reinterpret_cast<cudaStream_t>(stream));
}

int mslr_sampling(const int32_t N[3], int32_t Nc, int32_t Nt, const void* ksp, int64_t* K, int32_t* idx,
                  void* y, int64_t K_cap, void* stream) {
  if (!N || !ksp || !K || Nc <= 0 || Nt <= 0 || N[0] <= 0 || N[1] <= 0 || N[2] <= 0)
    return fail(MSLR_ERR_ARG, "bad argument");
  const int n3[3] = {N[0], N[1], N[2]};
  return sampling(n3, Nc, Nt, reinterpret_cast<const cf*>(ksp), K, idx, reinterpret_cast<cf*>(y), K_cap,
                  reinterpret_cast<cudaStream_t>(stream));
}

int mslr_prepare(mslr_ctx* ctx, const void* ksp, const void* smaps_raw, void* smaps_out, void* y_out,
                 int32_t* idx_out, double* scale_factor, void* stream) {
  CTX_CHECK(ctx);
  if (!ksp || !smaps_raw || !smaps_out || !y_out || !idx_out || !scale_factor)
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cf* smaps = reinterpret_cast<cf*>(smaps_out);
  cf* y = reinterpret_cast<cf*>(y_out);
  CTX_RET(ctx, sos_normalize(ctx->N, ctx->Nc, reinterpret_cast<const cf*>(smaps_raw), smaps, st));
  int64_t K = 0;
  CTX_RET(ctx, sampling(ctx->N, ctx->Nc, ctx->Nt, reinterpret_cast<const cf*>(ksp), &K, idx_out, y,
                        ctx->K, st));
  if (K != ctx->K)
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "the k-space has " + std::to_string(K) +
                                                " samples per frame, the context " +
                                                std::to_string(ctx->K)));
  CTX_RET(ctx, sense_bind(ctx, smaps, y, idx_out, 0, st));
  CTX_RET(ctx, prepare_scale(ctx, smaps, y, idx_out, scale_factor, st));
  return MSLR_OK;
}

int mslr_set_lambdas(mslr_ctx* ctx, const double* lambdas) {
  CTX_CHECK(ctx);
  if (!lambdas) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, set_lambdas(ctx, lambdas));
  return MSLR_OK;
}

int mslr_get_lambdas(const mslr_ctx* ctx, double* lambdas) {
  CTX_CHECK(ctx);
  if (!lambdas) return fail(MSLR_ERR_ARG, "null argument");
  for (int k = 0; k < ctx->Ns; ++k) lambdas[k] = ctx->lambdas[k];
  return MSLR_OK;
}

int mslr_pogm_grad(mslr_ctx* ctx, const void* X_true, int32_t niter, double L, double restart_cutoff,
                   double bsig, void* X, double* loss, double* grad_loglam, uint8_t* restarts_host,
                   void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!X_true || !X || !loss || !grad_loglam) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "null argument"));
  CTX_RET(ctx, check_pogm_args(ctx, niter, L, restart_cutoff, bsig));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  CTX_RET(ctx, pogm_grad(ctx, reinterpret_cast<const cf*>(X_true), niter, L, restart_cutoff, bsig,
                         reinterpret_cast<cf*>(X), loss, grad_loglam, restarts_host, st));
  CTX_RET(ctx, take_error(ctx, st));
  return MSLR_OK;
}

int mslr_cost(mslr_ctx* ctx, const void* X, int32_t ns_in, double* dc_cost, double* reg_cost,
              void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!X || ns_in <= 0) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad argument"));
  if (reg_cost && ns_in != ctx->Ns)
    return ctx_fail(ctx, fail(MSLR_ERR_ARG, "reg_cost needs one image per scale (ns_in == n_scales)"));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const cf* Xc = reinterpret_cast<const cf*>(X);
  if (dc_cost) CTX_RET(ctx, dc_cost_eval(ctx, Xc, ns_in, dc_cost, st));
  if (reg_cost) CTX_RET(ctx, patch_nucnorm_all(ctx, Xc, reg_cost, st));
  CTX_RET(ctx, take_error(ctx, st));
  return MSLR_OK;
}

int mslr_sync(mslr_ctx* ctx, void* stream) {
  CTX_CHECK(ctx);
  CTX_RET(ctx, take_error(ctx, reinterpret_cast<cudaStream_t>(stream)));
  return MSLR_OK;
}

int mslr_set_wait_limit(mslr_ctx* ctx, int64_t polls) {
  if (polls < 0 || polls > 0x7fffffff) {
    const int rc = fail(MSLR_ERR_ARG, "polls must be in [0, 2^31 - 1]");
    return ctx ? ctx_fail(ctx, rc) : rc;
  }
  if (!ctx) {
    set_context_free_polls((int)polls);
    return MSLR_OK;
  }
  if (ctx->wait_polls != (int)polls && ctx->gexec) {
    // the captured iteration holds the old limit in its kernel arguments
    cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
  }
  ctx->wait_polls = (int)polls;
  return MSLR_OK;
}

int mslr_set_graph(mslr_ctx* ctx, int32_t enable) {
  CTX_CHECK(ctx);
  ctx->use_graph = enable != 0;
  return MSLR_OK;
}

int mslr_launch_count(const mslr_ctx* ctx, uint64_t* count) {
  CTX_CHECK(ctx);
  if (!count) return fail(MSLR_ERR_ARG, "null output pointer");
  *count = ctx->launches;
  return MSLR_OK;
}

int mslr_power_iter(mslr_ctx* ctx, int32_t niter, double tol, double* sigma1, int32_t* iters_done,
                    void* stream) {
  CTX_CHECK(ctx);
  NEED_BOUND(ctx);
  if (!sigma1 || niter <= 0 || !(tol >= 0)) return ctx_fail(ctx, fail(MSLR_ERR_ARG, "bad argument"));
  int it = 0;
  CTX_RET(ctx, power_iter(ctx, niter, tol, sigma1, &it, reinterpret_cast<cudaStream_t>(stream)));
  CTX_RET(ctx, take_error(ctx, reinterpret_cast<cudaStream_t>(stream)));
  if (iters_done) *iters_done = it;
  return MSLR_OK;
}

}  // extern "C"
