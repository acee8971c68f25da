// pogm.cu — POGM with gradient restart and power iteration on sm_100a.
//
// pogm_mod (src/mirt_mod.jl:74-188) with mom=:pogm, μ=0, restart=:gr, as
// driven by run_recon (scripts/reconstruct.jl:220-226).  run_recon's g_prox
// writes into its argument (scripts/reconstruct.jl:196-202), so in the
// reference xnew aliases znew; consequently Fgrad ≡ fgrad, ynew ≡ unew and
// the β·α/ζold·(xold − zold) term is identically zero.  The recurrence run
// here is therefore, per iteration i (t_0 = 1, u_0 = x_0):
//
//   g   = ∇f(x_{i-1})                         (the same for every scale)
//   u_i = x_{i-1} − α g
//   t_i = ½(1 + √(1 + 4 t²))  (8 t² at i = niter);  β = (t−1)/t_i;  γ = σ t/t_i
//   z_i = u_i + β (u_i − u_{i-1}) + γ (u_i − x_{i-1});  ζ = α (1 + β + γ)
//   x_i = prox_{ζ Σ λ_k ‖·‖_*}(z_i)          (per-scale patch SVST)
//   restart if Σ Re(−g·(u_i − u_{i-1})) ≤ cutoff·‖g‖·‖u_i − u_{i-1}‖
//     (src/mirt_mod.jl:26-29: unconjugated product, Float64 sum)
//
// One fused kernel produces u_i and z_i and the FP64 restart reductions in a
// single pass over x, u and g; the scalar recurrence runs on the device so
// that a whole iteration can be replayed from a CUDA graph.
#include <cmath>
#include <cstring>
#include <vector>

#include <string>

#include "internal.h"

namespace mslr {

namespace {

constexpr int kRedBlocks = 1184;  // 148 SMs × 8 — fixed so reductions are deterministic
constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];
  }
  return r;  // valid in thread 0
}

// t, β, γ, ζ of the coming iteration (src/mirt_mod.jl:138-156).
__global__ void k_pogm_prepare(PogmState* s, double* thr) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double told = s->told;
  const double tnew = (s->iter == s->niter) ? 0.5 * (1.0 + sqrt(1.0 + 8.0 * told * told))
                                            : 0.5 * (1.0 + sqrt(1.0 + 4.0 * told * told));
  const double beta = (told - 1.0) / tnew;
  const double gamma = s->sig * told / tnew;
  s->tnew = tnew;
  s->beta = beta;
  s->gamma = gamma;
  s->zeta = s->alpha * (1.0 + beta + gamma);
  *thr = s->zeta;
}

// u ← x − α g;  z ← u + β(u − uold) + γ(u − x);  FP64 partial reductions.
__global__ void __launch_bounds__(kRedThreads)
    k_pogm_update(const cf* __restrict__ X, cf* __restrict__ U, const cf* __restrict__ G,
                  cf* __restrict__ Gold, cf* __restrict__ Z, int64_t E, int ns,
                  const PogmState* __restrict__ s, double* __restrict__ part) {
  __shared__ double sh[32];
  const float alpha = (float)s->alpha, beta = (float)s->beta, gamma = (float)s->gamma;
  const bool sigtest = (s->flags & 1) != 0;
  double r_dot = 0.0, r_g2 = 0.0, r_d2 = 0.0, r_sig = 0.0;
  // one element: g, and x/u of every scale at offset e
  auto one = [&](const cf g, const cf* xo, const cf* uo, cf* un, cf* zn) {
    const cf u = make_float2(xo->x - alpha * g.x, xo->y - alpha * g.y);
    const cf du = csub(u, *uo);
    *zn = make_float2(u.x + beta * du.x + gamma * (u.x - xo->x), u.y + beta * du.y + gamma * (u.y - xo->y));
    *un = u;
    r_dot += -((double)g.x * du.x - (double)g.y * du.y);
    r_d2 += (double)du.x * du.x + (double)du.y * du.y;
  };
  // pairs of elements with 16-byte accesses when every scale's slab starts on a
  // 16-byte boundary (E even and the caller's X 16-byte aligned; the library's
  // own buffers are), else element by element
  const bool vec = (E % 2 == 0) && ((reinterpret_cast<uintptr_t>(X) & 15u) == 0);
  const int64_t E2 = vec ? E / 2 : 0;
  const float4* G4 = reinterpret_cast<const float4*>(G);
  if (ns == 2) {   // two scales: every load of a pair issued before its stores
    const float4* X4 = reinterpret_cast<const float4*>(X);
    float4* U4 = reinterpret_cast<float4*>(U);
    float4* Z4 = reinterpret_cast<float4*>(Z);
    float4* GO4 = reinterpret_cast<float4*>(Gold);
    for (int64_t e2 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e2 < E2;
         e2 += (int64_t)gridDim.x * blockDim.x) {
      const int64_t o1 = E2 + e2;
      const float4 g4 = G4[e2];
      const float4 xa = X4[e2], ua = U4[e2], xb = X4[o1], ub = U4[o1];
      const float4 go = sigtest ? GO4[e2] : make_float4(0.f, 0.f, 0.f, 0.f);
      const cf g0 = make_float2(g4.x, g4.y), g1 = make_float2(g4.z, g4.w);
      r_g2 += (double)g0.x * g0.x + (double)g0.y * g0.y;
      r_g2 += (double)g1.x * g1.x + (double)g1.y * g1.y;
      if (sigtest) {
        r_sig += (double)g0.x * go.x - (double)g0.y * go.y;
        r_sig += (double)g1.x * go.z - (double)g1.y * go.w;
        GO4[e2] = g4;
      }
      cf un0, un1, zn0, zn1;
      {
        const cf x0 = make_float2(xa.x, xa.y), x1 = make_float2(xa.z, xa.w);
        const cf u0 = make_float2(ua.x, ua.y), u1 = make_float2(ua.z, ua.w);
        one(g0, &x0, &u0, &un0, &zn0);
        one(g1, &x1, &u1, &un1, &zn1);
        U4[e2] = make_float4(un0.x, un0.y, un1.x, un1.y);
        Z4[e2] = make_float4(zn0.x, zn0.y, zn1.x, zn1.y);
      }
      {
        const cf x0 = make_float2(xb.x, xb.y), x1 = make_float2(xb.z, xb.w);
        const cf u0 = make_float2(ub.x, ub.y), u1 = make_float2(ub.z, ub.w);
        one(g0, &x0, &u0, &un0, &zn0);
        one(g1, &x1, &u1, &un1, &zn1);
        U4[o1] = make_float4(un0.x, un0.y, un1.x, un1.y);
        Z4[o1] = make_float4(zn0.x, zn0.y, zn1.x, zn1.y);
      }
    }
  }
  for (int64_t e2 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; ns != 2 && e2 < E2;
       e2 += (int64_t)gridDim.x * blockDim.x) {
    const float4 g4 = G4[e2];
    const cf g0 = make_float2(g4.x, g4.y), g1 = make_float2(g4.z, g4.w);
    r_g2 += (double)g0.x * g0.x + (double)g0.y * g0.y;
    r_g2 += (double)g1.x * g1.x + (double)g1.y * g1.y;
    if (sigtest) {
      float4* GO4 = reinterpret_cast<float4*>(Gold);
      const float4 go = GO4[e2];
      r_sig += (double)g0.x * go.x - (double)g0.y * go.y;
      r_sig += (double)g1.x * go.z - (double)g1.y * go.w;
      GO4[e2] = g4;
    }
    for (int k = 0; k < ns; ++k) {
      const int64_t o2 = (int64_t)k * (E / 2) + e2;
      const float4 x4 = reinterpret_cast<const float4*>(X)[o2];
      const float4 u4 = reinterpret_cast<const float4*>(U)[o2];
      const cf x0 = make_float2(x4.x, x4.y), x1 = make_float2(x4.z, x4.w);
      const cf u0 = make_float2(u4.x, u4.y), u1 = make_float2(u4.z, u4.w);
      cf un0, un1, zn0, zn1;
      one(g0, &x0, &u0, &un0, &zn0);
      one(g1, &x1, &u1, &un1, &zn1);
      reinterpret_cast<float4*>(U)[o2] = make_float4(un0.x, un0.y, un1.x, un1.y);
      reinterpret_cast<float4*>(Z)[o2] = make_float4(zn0.x, zn0.y, zn1.x, zn1.y);
    }
  }
  for (int64_t e = (vec ? E : 0) + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
       e += (int64_t)gridDim.x * blockDim.x) {   // element by element when not vectorised
    const cf g = G[e];
    r_g2 += (double)g.x * g.x + (double)g.y * g.y;
    if (sigtest) {
      const cf go = Gold[e];
      r_sig += (double)g.x * go.x - (double)g.y * go.y;
      Gold[e] = g;
    }
    for (int k = 0; k < ns; ++k) {
      const int64_t o = (int64_t)k * E + e;
      const cf xo = X[o], uo = U[o];
      one(g, &xo, &uo, &U[o], &Z[o]);
    }
  }
  double v;
  v = block_sum(r_dot, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 4 + 0] = v;
  v = block_sum(r_g2, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 4 + 1] = v;
  v = block_sum(r_d2, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 4 + 2] = v;
  v = block_sum(r_sig, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 4 + 3] = v;
}

// Restart decision and t/σ update (src/mirt_mod.jl:163-184) from the
// iteration's totals tot = (Σ Re(−g·Δu), Σ|g|², Σ|Δu|², Σ Re(g·gold)).
__device__ void pogm_decide(PogmState* s, const double* tot, int ns, uint8_t* restarts, int32_t* err) {
  const double dot = tot[0];
  const double gnorm = sqrt((double)ns * tot[1]);   // ‖Fgrad‖ of the replicated 5-D gradient
  const double dnorm = sqrt(tot[2]);
  const double sigdot = (double)ns * tot[3];
  for (int q = 0; q < 4; ++q) s->red[q] = tot[q];
  if (!isfinite(dot) || !isfinite(gnorm) || !isfinite(dnorm)) atomicOr(err, kErrNonfinite);
  int restart = 0;
  double tnew = s->tnew;
  if (dot <= s->restart_cutoff * gnorm * dnorm) {
    tnew = 1.0;
    s->sig = 1.0;
    restart = 1;
  } else if ((s->flags & 1) && sigdot < 0.0) {
    s->sig = s->bsig * s->sig;
  }
  restarts[s->iter] = (uint8_t)restart;
  s->told = tnew;
  s->iter += 1;
}

// The partial sums of k_pogm_update's blocks added in block order.
__device__ void pogm_totals(const double* __restrict__ part, int nblocks, double* sh, double* tot) {
  double acc[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int q = 0; q < 4; ++q) acc[q] += part[b * 4 + q];
  for (int q = 0; q < 4; ++q) tot[q] = block_sum(acc[q], sh);
}

__global__ void k_pogm_finish(PogmState* s, const double* __restrict__ part, int nblocks,
                              int ns, uint8_t* restarts, int32_t* err) {
  __shared__ double sh[32];
  double tot[4];
  pogm_totals(part, nblocks, sh, tot);
  if (threadIdx.x == 0) pogm_decide(s, tot, ns, restarts, err);
}

// Sharded iteration: this rank's totals into sums (4 doubles, device), to be
// added over the ranks by the caller before k_pogm_decide_sums.
__global__ void k_pogm_reduce(const double* __restrict__ part, int nblocks, double* sums) {
  __shared__ double sh[32];
  double tot[4];
  pogm_totals(part, nblocks, sh, tot);
  if (threadIdx.x == 0)
    for (int q = 0; q < 4; ++q) sums[q] = tot[q];
}

__global__ void k_pogm_decide_sums(PogmState* s, const double* __restrict__ sums, int ns,
                                   uint8_t* restarts, int32_t* err) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double tot[4];
  for (int q = 0; q < 4; ++q) tot[q] = sums[q];
  pogm_decide(s, tot, ns, restarts, err);
}

__global__ void k_pogm_init(PogmState* s, double L, int niter, double cutoff, double bsig,
                            uint8_t* restarts) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  s->told = 1.0;
  s->sig = 1.0;
  s->tnew = 1.0;
  s->alpha = 1.0 / L;
  s->beta = s->gamma = 0.0;
  s->zeta = 1.0;
  s->restart_cutoff = cutoff;
  s->bsig = bsig;
  s->iter = 1;
  s->niter = niter;
  s->flags = (bsig != 1.0) ? 1 : 0;
  for (int q = 0; q < 4; ++q) s->red[q] = 0.0;
  restarts[0] = 0;
}

__global__ void k_set_scalar(double* dst, double v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = v;
}

// ---- power iteration helpers ----------------------------------------------
__global__ void k_fill_one(cf* x, int64_t E) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
       e += (int64_t)gridDim.x * blockDim.x)
    x[e] = make_float2(1.f, 0.f);
}

// part[b] = (Σ Re(conj(x)·p), Σ|x|², Σ|p|²)
__global__ void __launch_bounds__(kRedThreads)
    k_dots(const cf* __restrict__ x, const cf* __restrict__ p, int64_t E, double* part) {
  __shared__ double sh[32];
  double a = 0, b = 0, c = 0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
       e += (int64_t)gridDim.x * blockDim.x) {
    const cf u = x[e], v = p[e];
    a += (double)u.x * v.x + (double)u.y * v.y;
    b += (double)u.x * u.x + (double)u.y * u.y;
    c += (double)v.x * v.x + (double)v.y * v.y;
  }
  double r;
  r = block_sum(a, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 3 + 0] = r;
  r = block_sum(b, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 3 + 1] = r;
  r = block_sum(c, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 3 + 2] = r;
}

__global__ void k_scale_into(cf* __restrict__ x, const cf* __restrict__ p, float s, int64_t E) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
       e += (int64_t)gridDim.x * blockDim.x)
    x[e] = cscale(p[e], s);
}

// ---- pogm_mod's other options (mom = :pgm / :fpgm, restart = :none / :fr, μ > 0) ----
// Z[k] = X[k] − α g for every scale k (the gradient step, the same g for all)
__global__ void k_grad_step(const cf* __restrict__ X, const cf* __restrict__ G, float alpha,
                            cf* __restrict__ Z, int64_t E, int ns) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
       e += (int64_t)gridDim.x * blockDim.x) {
    const cf g = G[e];
    for (int k = 0; k < ns; ++k) {
      const cf x = X[(int64_t)k * E + e];
      Z[(int64_t)k * E + e] = make_float2(x.x - alpha * g.x, x.y - alpha * g.y);
    }
  }
}

// _gr_restart's sums for :pgm / :fpgm (src/mirt_mod.jl:26-29, :124-133):
// Fgrad = −(ynew − xold)/α, Δy = ynew − yold; partials of Σ Re(−Fgrad·Δy),
// ‖Fgrad‖², ‖Δy‖² over n elements (unconjugated product, FP64)
__global__ void __launch_bounds__(kRedThreads)
    k_pgm_sums(const cf* __restrict__ Yn, const cf* __restrict__ X, const cf* __restrict__ Yold,
               double inv_alpha, int64_t n, double* __restrict__ part) {
  __shared__ double sh[32];
  double r_dot = 0.0, r_f2 = 0.0, r_d2 = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const cf yn = Yn[e], xo = X[e], yo = Yold[e];
    const double fr = -((double)yn.x - xo.x) * inv_alpha, fi = -((double)yn.y - xo.y) * inv_alpha;
    const double dr = (double)yn.x - yo.x, di = (double)yn.y - yo.y;
    r_dot += -(fr * dr - fi * di);
    r_f2 += fr * fr + fi * fi;
    r_d2 += dr * dr + di * di;
  }
  double v;
  v = block_sum(r_dot, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 4 + 0] = v;
  v = block_sum(r_f2, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 4 + 1] = v;
  v = block_sum(r_d2, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x * 4 + 2] = v;
    part[blockIdx.x * 4 + 3] = 0.0;
  }
}

// X = Yn + β (Yn − Yold) over n elements (:fpgm's momentum step)
__global__ void k_extrapolate(cf* __restrict__ X, const cf* __restrict__ Yn, const cf* __restrict__ Yold,
                              float beta, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const cf yn = Yn[e], yo = Yold[e];
    X[e] = make_float2(yn.x + beta * (yn.x - yo.x), yn.y + beta * (yn.y - yo.y));
  }
}

}  // namespace

int set_scalar(double* dst, double v, cudaStream_t st) {
  k_set_scalar<<<1, 32, 0, st>>>(dst, v);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int pogm_setup(Ctx* c) {
  int rc;
  const size_t E = (size_t)c->Nt * c->nvox;
  if ((rc = dalloc(c, (void**)&c->d_U, (size_t)c->Ns * E * sizeof(cf)))) return rc;
  if ((rc = dalloc(c, (void**)&c->d_Z, (size_t)c->Ns * E * sizeof(cf)))) return rc;
  if ((rc = dalloc(c, (void**)&c->d_G, E * sizeof(cf)))) return rc;
  if ((rc = dalloc(c, (void**)&c->d_part, (size_t)kRedBlocks * 4 * sizeof(double)))) return rc;
  if ((rc = dalloc(c, (void**)&c->d_state, sizeof(PogmState)))) return rc;
  c->nred_blocks = kRedBlocks;
  return MSLR_OK;
}

int init_x0(Ctx* c, cf* X, cudaStream_t st) {
  const size_t E = (size_t)c->Nt * c->nvox;
  MSLR_CUDA_TRY(cudaMemcpyAsync(X, c->d_ahy, E * sizeof(cf), cudaMemcpyDeviceToDevice, st));
  if (c->Ns > 1)
    MSLR_CUDA_TRY(cudaMemsetAsync(X + E, 0, (size_t)(c->Ns - 1) * E * sizeof(cf), st));
  return MSLR_OK;
}

int pogm_begin(Ctx* c, cf* X, int niter, double L, double cutoff, double bsig, cudaStream_t st) {
  int rc;
  const size_t E = (size_t)c->Nt * c->nvox;
  if (niter + 1 > c->restarts_cap) {
    if (c->d_restarts) cudaFree(c->d_restarts);
    c->d_restarts = nullptr;
    if ((rc = dalloc(c, (void**)&c->d_restarts, (size_t)niter + 1))) return rc;
    c->restarts_cap = niter + 1;
  }
  MSLR_CUDA_TRY(cudaMemsetAsync(c->d_restarts, 0, (size_t)niter + 1, st));
  if (bsig != 1.0) {
    if (!c->d_Gold && (rc = dalloc(c, (void**)&c->d_Gold, E * sizeof(cf)))) return rc;
    MSLR_CUDA_TRY(cudaMemsetAsync(c->d_Gold, 0, E * sizeof(cf), st));
  }
  // u_0 = x_0 (src/mirt_mod.jl:98)
  MSLR_CUDA_TRY(cudaMemcpyAsync(c->d_U, X, (size_t)c->Ns * E * sizeof(cf),
                                cudaMemcpyDeviceToDevice, st));
  k_pogm_init<<<1, 32, 0, st>>>(c->d_state, L, niter, cutoff, bsig, c->d_restarts);
  MSLR_CUDA_TRY(cudaGetLastError());
  c->pogm_ready = true;
  return MSLR_OK;
}

static int pogm_step_body(Ctx* c, cf* X, cudaStream_t st) {
  int rc;
  const int64_t E = (int64_t)c->Nt * c->nvox;
  // 1. g = A'(A Σ_k x_k − y)   (scripts/reconstruct.jl:180-183)
  if ((rc = normal_op(c, X, c->Ns, E, c->d_G, true, st))) return rc;
  // 2. momentum scalars, 3. fused u/z update + restart reductions
  k_pogm_prepare<<<1, 32, 0, st>>>(c->d_state, c->d_thr);
  k_pogm_update<<<kRedBlocks, kRedThreads, 0, st>>>(X, c->d_U, c->d_G, c->d_Gold, c->d_Z, E,
                                                    c->Ns, c->d_state, c->d_part);
  k_pogm_finish<<<1, kRedThreads, 0, st>>>(c->d_state, c->d_part, kRedBlocks, c->Ns,
                                           c->d_restarts, c->d_err);
  MSLR_CUDA_TRY(cudaGetLastError());
  c->launches += 3;
  // 4. x_i = g_prox(z_i, ζ): patch SVST with threshold ζ·λ_k — scale after
  //    scale in the plain form, all scales batched in the tuned form
  if (c->tuned()) return patch_svst_all(c, c->d_thr, c->d_Z, X, st);
  for (int k = 0; k < c->Ns; ++k) {
    if ((rc = patch_svst(c, k, c->d_thr, c->lambdas[k], c->d_Z + k * E, X + k * E, st)))
      return rc;
  }
  return MSLR_OK;
}

// Sharded iteration, first half on this rank's frames: g = A'(A Σ_k x_k − y),
// the momentum scalars, u and z (z into Zout, (Ns, Nt, nvox) of this
// context's frames) and this rank's restart totals into sums_dev (4 doubles).
// The caller adds sums_dev over the ranks, then calls pogm_step_decide.
int pogm_step_local(Ctx* c, cf* X, cf* Zout, double* sums_dev, cudaStream_t st) {
  int rc;
  const int64_t E = (int64_t)c->Nt * c->nvox;
  if ((rc = normal_op(c, X, c->Ns, E, c->d_G, true, st))) return rc;
  k_pogm_prepare<<<1, 32, 0, st>>>(c->d_state, c->d_thr);
  k_pogm_update<<<kRedBlocks, kRedThreads, 0, st>>>(X, c->d_U, c->d_G, c->d_Gold, Zout, E, c->Ns,
                                                    c->d_state, c->d_part);
  k_pogm_reduce<<<1, kRedThreads, 0, st>>>(c->d_part, kRedBlocks, sums_dev);
  MSLR_CUDA_TRY(cudaGetLastError());
  c->launches += 3;
  return MSLR_OK;
}

// Restart decision and t/σ update of a sharded iteration from the totals
// over all ranks.
int pogm_step_decide(Ctx* c, const double* sums_dev, cudaStream_t st) {
  k_pogm_decide_sums<<<1, 32, 0, st>>>(c->d_state, sums_dev, c->Ns, c->d_restarts, c->d_err);
  MSLR_CUDA_TRY(cudaGetLastError());
  c->launches += 1;
  return MSLR_OK;
}

// α, β, γ, ζ of the current iteration (after pogm_step_local).  Synchronises st.
int pogm_scalars(Ctx* c, double* out, cudaStream_t st) {
  PogmState h;
  MSLR_CUDA_TRY(cudaMemcpyAsync(&h, c->d_state, sizeof(PogmState), cudaMemcpyDeviceToHost, st));
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  out[0] = h.alpha;
  out[1] = h.beta;
  out[2] = h.gamma;
  out[3] = h.zeta;
  return MSLR_OK;
}

// One POGM iteration.  In the tuned form the whole iteration (about 1400
// kernels at 90×90×60) is captured once into a CUDA graph on the context's
// private stream and replayed; the caller's stream is joined with events on
// both sides, so any stream (the legacy default included) may be passed.  All
// per-iteration scalars live in device memory (PogmState), so one graph
// serves every iteration of every run on the same X.
int pogm_step(Ctx* c, cf* X, cudaStream_t st) {
  if (!c->tuned() || !c->use_graph) return pogm_step_body(c, X, st);
  if (!c->gstream) {
    MSLR_CUDA_TRY(cudaStreamCreateWithFlags(&c->gstream, cudaStreamNonBlocking));
    MSLR_CUDA_TRY(cudaEventCreateWithFlags(&c->gev_in, cudaEventDisableTiming));
    MSLR_CUDA_TRY(cudaEventCreateWithFlags(&c->gev_out, cudaEventDisableTiming));
  }
  if (!c->gexec || c->gX != X) {
    if (c->gexec) {
      cudaGraphExecDestroy(c->gexec);
      c->gexec = nullptr;
    }
    const uint64_t l0 = c->launches;
    MSLR_CUDA_TRY(cudaStreamBeginCapture(c->gstream, cudaStreamCaptureModeThreadLocal));
    const int rc = pogm_step_body(c, X, c->gstream);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->gstream, &g);
    if (rc || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      c->launches = l0;
      return rc ? rc : fail(MSLR_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    }
    const cudaError_t ei = cudaGraphInstantiate(&c->gexec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      c->gexec = nullptr;
      c->launches = l0;
      return fail(MSLR_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    }
    c->glaunches = c->launches - l0;
    c->launches = l0;
    c->gX = X;
  }
  MSLR_CUDA_TRY(cudaEventRecord(c->gev_in, st));
  MSLR_CUDA_TRY(cudaStreamWaitEvent(c->gstream, c->gev_in, 0));
  MSLR_CUDA_TRY(cudaGraphLaunch(c->gexec, c->gstream));
  MSLR_CUDA_TRY(cudaEventRecord(c->gev_out, c->gstream));
  MSLR_CUDA_TRY(cudaStreamWaitEvent(st, c->gev_out, 0));
  c->launches += c->glaunches;
  return MSLR_OK;
}

int power_iter(Ctx* c, int niter, double tol, double* sigma1, int* iters, cudaStream_t st) {
  int rc;
  const int64_t E = (int64_t)c->Nt * c->nvox;
  cf* x = c->d_U;   // scratch: first scale slot of u
  cf* p = c->d_G;
  std::vector<double> h(kRedBlocks * 3);
  auto dots = [&](double* out) -> int {
    k_dots<<<kRedBlocks, kRedThreads, 0, st>>>(x, p, E, c->d_part);
    MSLR_CUDA_TRY(cudaGetLastError());
    MSLR_CUDA_TRY(cudaMemcpyAsync(h.data(), c->d_part, h.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    MSLR_CUDA_TRY(cudaStreamSynchronize(st));
    out[0] = out[1] = out[2] = 0;
    for (int b = 0; b < kRedBlocks; ++b)
      for (int q = 0; q < 3; ++q) out[q] += h[b * 3 + q];
    return MSLR_OK;
  };
  k_fill_one<<<kRedBlocks, kRedThreads, 0, st>>>(x, E);   // x0 = ones (src/mirt_mod.jl:219)
  double ratio_old = INFINITY;
  int it = 0;
  double d[3];
  for (it = 1; it <= niter; ++it) {
    if ((rc = normal_op(c, x, 1, E, p, false, st))) return rc;   // p = A'A x
    if ((rc = dots(d))) return rc;
    // ‖Ax‖/‖x‖ with ‖Ax‖² = <x, A'A x>
    const double ratio = std::sqrt(std::max(d[0], 0.0)) / std::sqrt(d[1]);
    if (!std::isfinite(ratio)) return fail(MSLR_ERR_NONFINITE, "power iteration diverged");
    if (std::fabs(ratio - ratio_old) / ratio < tol) break;
    ratio_old = ratio;
    // x = A'Ax / ‖A'Ax‖
    k_scale_into<<<kRedBlocks, kRedThreads, 0, st>>>(x, p, (float)(1.0 / std::sqrt(d[2])), E);
  }
  if (iters) *iters = std::min(it, niter);
  if ((rc = normal_op(c, x, 1, E, p, false, st))) return rc;
  if ((rc = dots(d))) return rc;
  *sigma1 = std::sqrt(std::max(d[0], 0.0)) / std::sqrt(d[1]);
  return MSLR_OK;
}

}  // namespace mslr

namespace mslr {

// The four totals of the reduction partials in d_part, to the host.
static int totals_to_host(Ctx* c, double* tot, double* d_tot, cudaStream_t st) {
  k_pogm_reduce<<<1, kRedThreads, 0, st>>>(c->d_part, kRedBlocks, d_tot);
  MSLR_CUDA_TRY(cudaGetLastError());
  MSLR_CUDA_TRY(cudaMemcpyAsync(tot, d_tot, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  c->launches += 1;
  return MSLR_OK;
}

// g_prox of run_recon (scripts/reconstruct.jl:196-202) with threshold c·λ_k
static int prox_all(Ctx* c, double cthr, const cf* Zin, cf* Xout, cudaStream_t st) {
  int rc;
  if ((rc = set_scalar(c->d_thr, cthr, st))) return rc;
  if (c->tuned()) return patch_svst_all(c, c->d_thr, Zin, Xout, st);
  const int64_t E = (int64_t)c->Nt * c->nvox;
  for (int k = 0; k < c->Ns; ++k)
    if ((rc = patch_svst(c, k, c->d_thr, c->lambdas[k], Zin + k * E, Xout + k * E, st))) return rc;
  return MSLR_OK;
}

// run_recon's comp_cost = dc_cost + reg_cost of X (scripts/reconstruct.jl:176-194)
static int fcost(Ctx* c, const cf* X, double* out, cudaStream_t st) {
  double dc = 0.0, reg = 0.0;
  int rc;
  if ((rc = dc_cost_eval(c, X, c->Ns, &dc, st))) return rc;
  if ((rc = patch_nucnorm_all(c, X, &reg, st))) return rc;
  *out = dc + reg;
  return MSLR_OK;
}

// pogm_mod (src/mirt_mod.jl:74-188) with any of its options and run_recon's
// closures, on the host loop (one synchronisation per iteration): mom 0 =
// :pgm, 1 = :fpgm, 2 = :pogm; restart 0 = :none, 1 = :gr, 2 = :fr; f_mu ≥ 0.
// X holds x0 on entry and pogm_mod's return value on exit (xnew for :pogm,
// ynew otherwise).  restarts_h (niter + 1) receives the logger's flags.
int pogm_run_options(Ctx* c, cf* X, int niter, double L, double mu, int mom, int restart,
                     double cutoff, double bsig, uint8_t* restarts_h, cudaStream_t st) {
  int rc;
  const int64_t E = (int64_t)c->Nt * c->nvox;
  const int64_t n = (int64_t)c->Ns * E;
  const size_t bytes = (size_t)n * sizeof(cf);
  const double q = mu / L;
  double* d_tot = c->d_thr + 8;   // 4 doubles of the context's scalar slots
  std::vector<uint8_t> flags((size_t)niter + 1, 0);
  double told = 1.0, sig = 1.0, Fcostold = 0.0;
  if (restart == 2 && (rc = fcost(c, X, &Fcostold, st))) return rc;
  if (mom != 2) {
    // :pgm / :fpgm — yold in U, the prox input in Z, ynew in the second half of Z's
    // neighbour buffer: X (xold), U (yold), Z (x − α g), Yn (ynew)
    if (!c->d_Y && (rc = dalloc(c, (void**)&c->d_Y, bytes))) return rc;
    cf* Yold = c->d_U;
    cf* Yn = c->d_Y;
    MSLR_CUDA_TRY(cudaMemcpyAsync(Yold, X, bytes, cudaMemcpyDeviceToDevice, st));
    for (int it = 1; it <= niter; ++it) {
      const double alpha = (mom == 0 && mu != 0.0) ? 2.0 / (L + mu) : 1.0 / L;
      if ((rc = normal_op(c, X, c->Ns, E, c->d_G, true, st))) return rc;
      k_grad_step<<<kRedBlocks, kRedThreads, 0, st>>>(X, c->d_G, (float)alpha, c->d_Z, E, c->Ns);
      MSLR_CUDA_TRY(cudaGetLastError());
      c->launches += 1;
      if ((rc = prox_all(c, alpha, c->d_Z, Yn, st))) return rc;
      bool rs = false;
      if (restart != 0) {
        if (restart == 2) {
          double Fcostnew = 0.0;
          if ((rc = fcost(c, Yn, &Fcostnew, st))) return rc;
          rs = Fcostnew > Fcostold;
          Fcostold = Fcostnew;
        } else {
          k_pgm_sums<<<kRedBlocks, kRedThreads, 0, st>>>(Yn, X, Yold, 1.0 / alpha, n, c->d_part);
          MSLR_CUDA_TRY(cudaGetLastError());
          c->launches += 1;
          double tot[4];
          if ((rc = totals_to_host(c, tot, d_tot, st))) return rc;
          if (!std::isfinite(tot[0]) || !std::isfinite(tot[1]) || !std::isfinite(tot[2]))
            return fail(MSLR_ERR_NONFINITE, "non-finite value in the restart sums");
          rs = tot[0] <= cutoff * std::sqrt(tot[1]) * std::sqrt(tot[2]);
        }
        if (rs) told = 1.0;
      }
      flags[it] = rs ? 1 : 0;
      double tnew = told;
      if (mom == 1) {
        double beta;
        if (mu != 0.0) {
          beta = (1.0 - std::sqrt(q)) / (1.0 + std::sqrt(q));
        } else {
          tnew = 0.5 * (1.0 + std::sqrt(1.0 + 4.0 * told * told));
          beta = (told - 1.0) / tnew;
        }
        k_extrapolate<<<kRedBlocks, kRedThreads, 0, st>>>(X, Yn, Yold, (float)beta, n);
        MSLR_CUDA_TRY(cudaGetLastError());
        c->launches += 1;
      } else {
        MSLR_CUDA_TRY(cudaMemcpyAsync(X, Yn, bytes, cudaMemcpyDeviceToDevice, st));
      }
      std::swap(Yold, Yn);   // yold ← ynew
      if (mom != 0 && mu == 0.0) told = tnew;
    }
    // pogm_mod returns ynew for :pgm / :fpgm
    MSLR_CUDA_TRY(cudaMemcpyAsync(X, Yold, bytes, cudaMemcpyDeviceToDevice, st));
  } else {
    // :pogm with restart :none / :fr or μ > 0: the fused update of the default
    // path with the scalars of this iteration written from the host
    PogmState h{};
    h.alpha = 1.0 / L;
    h.flags = (bsig != 1.0 && restart != 0) ? 1 : 0;
    if (h.flags) {
      if (!c->d_Gold && (rc = dalloc(c, (void**)&c->d_Gold, (size_t)E * sizeof(cf)))) return rc;
      MSLR_CUDA_TRY(cudaMemsetAsync(c->d_Gold, 0, (size_t)E * sizeof(cf), st));
    }
    MSLR_CUDA_TRY(cudaMemcpyAsync(c->d_U, X, bytes, cudaMemcpyDeviceToDevice, st));   // uold = x0
    for (int it = 1; it <= niter; ++it) {
      double tnew = told, beta, gamma;
      if (mu != 0.0) {
        const double r = 2.0 + q - std::sqrt(q * q + 8.0 * q);
        beta = r * r / 4.0 / (1.0 - q);
        gamma = r / 2.0;
      } else {
        tnew = 0.5 * (1.0 + std::sqrt(1.0 + (it == niter ? 8.0 : 4.0) * told * told));
        beta = (told - 1.0) / tnew;
        gamma = sig * told / tnew;
      }
      h.beta = beta;
      h.gamma = gamma;
      MSLR_CUDA_TRY(cudaMemcpyAsync(c->d_state, &h, sizeof(PogmState), cudaMemcpyHostToDevice, st));
      if ((rc = normal_op(c, X, c->Ns, E, c->d_G, true, st))) return rc;
      k_pogm_update<<<kRedBlocks, kRedThreads, 0, st>>>(X, c->d_U, c->d_G, c->d_Gold, c->d_Z, E, c->Ns,
                                                        c->d_state, c->d_part);
      MSLR_CUDA_TRY(cudaGetLastError());
      c->launches += 1;
      double tot[4];
      if ((rc = totals_to_host(c, tot, d_tot, st))) return rc;
      const double zeta = h.alpha * (1.0 + beta + gamma);
      if ((rc = prox_all(c, zeta, c->d_Z, X, st))) return rc;
      bool rs = false;
      if (restart != 0) {
        if (restart == 2) {
          double Fcostnew = 0.0;
          if ((rc = fcost(c, X, &Fcostnew, st))) return rc;
          rs = Fcostnew > Fcostold;
          Fcostold = Fcostnew;
        } else {
          if (!std::isfinite(tot[0]) || !std::isfinite(tot[1]) || !std::isfinite(tot[2]))
            return fail(MSLR_ERR_NONFINITE, "non-finite value in the restart sums");
          rs = tot[0] <= cutoff * std::sqrt((double)c->Ns * tot[1]) * std::sqrt(tot[2]);
        }
        if (rs) {
          tnew = 1.0;
          sig = 1.0;
        } else if (h.flags && (double)c->Ns * tot[3] < 0.0) {
          sig = bsig * sig;
        }
      }
      flags[it] = rs ? 1 : 0;
      if (mu == 0.0) told = tnew;
    }
  }
  if (restarts_h) std::memcpy(restarts_h, flags.data(), flags.size());
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  return MSLR_OK;
}

}  // namespace mslr
