// grad.cu — reverse-mode gradient of the unrolled POGM with respect to the
// per-scale weights, d loss / d log λ_k, on sm_100a.
//
// The reference runs pogm_mod with run_recon's aliasing g_prox
// (src/mirt_mod.jl:74-188, scripts/reconstruct.jl:196-226) and does not
// differentiate it.  With the restart decisions and momentum scalars of a run
// held fixed, that iteration is (pogm.cu)
//     u_i = x_{i-1} − α ∇f(x_{i-1}),   ∇f(x) = R A'(A Σ_k x_k − y)
//     z_i = a_i u_i − β_i u_{i-1} − γ_i x_{i-1},   a_i = 1 + β_i + γ_i
//     x_i = prox_i(z_i)   (per scale k: patch SVST with threshold ζ_i λ_k)
// and for loss = ½ ‖Σ_k x_N,k − X_true‖² reverse accumulation runs, from
// x̄_N = R(Σ_k x_N,k − X_true), ū_N = 0, for i = N … 1:
//     z̄_i = J_prox(z_i)ᴴ x̄_i,   d loss/d log λ_k += ζ_i λ_k ∂loss/∂β
//     w    = ū_i + a_i z̄_i
//     x̄_{i-1} = w − α R A'A Σ_k w_k − γ_i z̄_i,   ū_{i-1} = −β_i z̄_i
// (A'A is self-adjoint and R, Σ are each other's adjoints).  The forward
// stores z_i for every iteration (checkpoints); the backward recomputes each
// patch's eigen-decomposition from them.
//
// Patch-SVST backward (Gram form, matching svst.cu's M / W conventions): for
// a patch's n × L matrix M with G = M Mᴴ = V Λ Vᴴ, W = V f(Λ) Vᴴ,
// f(λ) = max(1 − β/√λ, 0) and M_out = W M, the cotangent Ō of M_out gives
//     W̄ = Ō Mᴴ,   D = Vᴴ W̄ V,   E = F ⊙ (D + Dᴴ),   K = V E Vᴴ
//     M̄ = W Ō + K M,       ∂loss/∂β = Σ_i ∂f/∂β(λ_i) Re D_ii
// with F the divided differences of f (Daleckii–Krein).  Every product runs
// on the CUDA cores in FP32; the eigenpairs come from the eigen stage's full
// mode (FP64 bisection and twisted factorisation).
#include <cmath>
#include <vector>

#include "internal.h"
#include "patchmap.cuh"

namespace mslr {

namespace {

constexpr int kTile = 64;
constexpr int kKc = 16;
constexpr int kRedBlocks = 592;

__device__ __forceinline__ cf cmul_(cf a, cf b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// W̄[ip][a][b] = Σ_l Ō[a][l] conj(M[b][l]) over l in this split's chunk, Ō
// and M read through the patch map from two images.  Row-major n × n blocks,
// one per (split, patch) when split.  grid (T·T, Np, nsplit).
__global__ void __launch_bounds__(256) k_xgram(const cf* __restrict__ imgO, const cf* __restrict__ imgM,
                                               PatchMap m, cf* __restrict__ out, int nsplit, int lchunk) {
  __shared__ cf As[kKc][kTile + 1];
  __shared__ cf Bs[kKc][kTile + 1];
  const int T = (m.n + kTile - 1) / kTile;
  const int ta = blockIdx.x / T, tb = blockIdx.x - ta * T;
  const int64_t ip = blockIdx.y, np = gridDim.y;
  const int split = blockIdx.z;
  const int64_t org = patch_origin(m, ip);
  const int a0 = ta * kTile, b0 = tb * kTile;
  const int l_begin = split * lchunk;
  const int l_end = min(m.L, l_begin + lchunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  cf acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
  for (int l0 = l_begin; l0 < l_end; l0 += kKc) {
    for (int q = threadIdx.x; q < kKc * kTile; q += blockDim.x) {
      int kk, r;
      if (m.tall) {
        kk = q % kKc;
        r = q / kKc;
      } else {
        r = q % kTile;
        kk = q / kTile;
      }
      const int l = l0 + kk;
      cf va = make_float2(0.f, 0.f), vb = make_float2(0.f, 0.f);
      if (l < l_end) {
        if (a0 + r < m.n) va = m_elem(m, imgO, org, a0 + r, l);
        if (b0 + r < m.n) vb = m_elem(m, imgM, org, b0 + r, l);
      }
      As[kk][r] = va;
      Bs[kk][r] = vb;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kKc; ++kk) {
      cf av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x += av[i].x * bv[j].x + av[i].y * bv[j].y;
          acc[i][j].y += av[i].y * bv[j].x - av[i].x * bv[j].y;
        }
    }
    __syncthreads();
  }
  const int n = m.n;
  cf* Wb = out + ((int64_t)split * np + ip) * n * n;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int a = a0 + ty * 4 + i, b = b0 + tx * 4 + j;
      if (a < n && b < n) Wb[(int64_t)a * n + b] = acc[i][j];
    }
}

// out[e] = Σ_s part[s·total + e], splits in order
__global__ void k_split_sum(const cf* __restrict__ part, cf* __restrict__ out, int nsplit, int64_t total) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    cf s = part[e];
    for (int q = 1; q < nsplit; ++q) s = cadd(s, part[q * total + e]);
    out[e] = s;
  }
}

// C[ip] = op_a(A[ip]) · op_b(B[ip]) for row-major n × n blocks; op 0 = as is,
// 1 = conjugate transpose.  grid (T·T, Np), 256 threads, 4 × 4 per thread.
template <int OPA, int OPB>
__global__ void __launch_bounds__(256) k_bgemm(const cf* __restrict__ A, const cf* __restrict__ B,
                                               cf* __restrict__ C, int n) {
  __shared__ cf As[kKc][kTile + 1];   // As[k][i] = op_a(A)(i, k)
  __shared__ cf Bs[kKc][kTile + 1];   // Bs[k][j] = op_b(B)(k, j)
  const int T = (n + kTile - 1) / kTile;
  const int ti = blockIdx.x / T, tj = blockIdx.x - ti * T;
  const int64_t nn = (int64_t)n * n;
  const cf* Ap = A + blockIdx.y * nn;
  const cf* Bp = B + blockIdx.y * nn;
  const int i0 = ti * kTile, j0 = tj * kTile;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  cf acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
  for (int k0 = 0; k0 < n; k0 += kKc) {
    for (int q = threadIdx.x; q < kKc * kTile; q += blockDim.x) {
      {   // A: contiguous index fastest across threads
        int kk, r;
        if (OPA == 0) {   // A[i][k]: k contiguous
          kk = q % kKc;
          r = q / kKc;
        } else {          // conj(A[k][i]): i contiguous
          r = q % kTile;
          kk = q / kTile;
        }
        const int i = i0 + r, k = k0 + kk;
        cf v = make_float2(0.f, 0.f);
        if (i < n && k < n) v = (OPA == 0) ? Ap[(int64_t)i * n + k] : cconj(Ap[(int64_t)k * n + i]);
        As[kk][r] = v;
      }
      {
        int kk, r;
        if (OPB == 0) {   // B[k][j]: j contiguous
          r = q % kTile;
          kk = q / kTile;
        } else {          // conj(B[j][k]): k contiguous
          kk = q % kKc;
          r = q / kKc;
        }
        const int j = j0 + r, k = k0 + kk;
        cf v = make_float2(0.f, 0.f);
        if (j < n && k < n) v = (OPB == 0) ? Bp[(int64_t)k * n + j] : cconj(Bp[(int64_t)j * n + k]);
        Bs[kk][r] = v;
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kKc; ++kk) {
      cf av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x += av[i].x * bv[j].x - av[i].y * bv[j].y;
          acc[i][j].y += av[i].x * bv[j].y + av[i].y * bv[j].x;
        }
    }
    __syncthreads();
  }
  cf* Cp = C + blockIdx.y * nn;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int a = i0 + ty * 4 + i, b = j0 + tx * 4 + j;
      if (a < n && b < n) Cp[(int64_t)a * n + b] = acc[i][j];
    }
}

// One CTA per patch: E = F ⊙ (D + Dᴴ), T3 = V diag(f(λ)), and
// bbar[ip] = Σ_i ∂f/∂β(λ_i) Re D_ii.  F_ij = (f_i − f_j)/(λ_i − λ_j) in
// cancellation-free forms (both above β²: β / (s_i s_j (s_i + s_j)); one
// above: (s − β) / (s (s_a² − s_b²)) with s the one above; none: 0).
__global__ void __launch_bounds__(256) k_divdiff(const cf* __restrict__ D, const double* __restrict__ lam,
                                                 const cf* __restrict__ V, double beta, int n,
                                                 cf* __restrict__ E, cf* __restrict__ T3,
                                                 double* __restrict__ bbar) {
  __shared__ double red[32];
  const int64_t ip = blockIdx.x;
  const int64_t nn = (int64_t)n * n;
  const cf* Dp = D + ip * nn;
  const double* lp = lam + ip * n;
  const cf* Vp = V + ip * nn;
  cf* Ep = E + ip * nn;
  cf* Tp = T3 + ip * nn;
  for (int64_t q = threadIdx.x; q < nn; q += blockDim.x) {
    const int i = (int)(q / n), j = (int)(q - (int64_t)i * n);
    const double si = sqrt(fmax(lp[i], 0.0)), sj = sqrt(fmax(lp[j], 0.0));
    const bool ai = si > beta, aj = sj > beta;
    double F = 0.0;
    if (ai && aj) F = beta / (si * sj * (si + sj));
    else if (ai) F = (si - beta) / (si * (si - sj) * (si + sj));
    else if (aj) F = (sj - beta) / (sj * (sj - si) * (si + sj));
    const cf dij = Dp[q], dji = Dp[(int64_t)j * n + i];
    Ep[q] = make_float2((float)(F * ((double)dij.x + dji.x)), (float)(F * ((double)dij.y - dji.y)));
    const float fj = aj ? (float)(1.0 - beta / sj) : 0.f;
    Tp[q] = make_float2(Vp[q].x * fj, Vp[q].y * fj);
  }
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double si = sqrt(fmax(lp[i], 0.0));
    if (si > beta) s += -(double)Dp[(int64_t)i * n + i].x / si;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    bbar[ip] = t;
  }
}

// P̄ = (W Ō + K M) in the image domain (svst.cu's k_rebuild with two terms):
//   tall: out[t=a][vox_l] = Σ_b conj(W[a][b]) x̄[b][vox_l] + conj(K[a][b]) z[b][vox_l]
//   wide: out[t=l][vox_a] = Σ_b W[a][b] x̄[l][vox_b] + K[a][b] z[l][vox_b]
// W, K row-major n × n per patch.  grid (ceil(n/64), ceil(L/64), Np).
__global__ void __launch_bounds__(256) k_vjp_rebuild(const cf* __restrict__ xb, const cf* __restrict__ z,
                                                     const cf* __restrict__ W, const cf* __restrict__ K,
                                                     PatchMap m, cf* __restrict__ out, int direct) {
  __shared__ cf As[kKc][kTile + 1];
  __shared__ cf Bs[kKc][kTile + 1];
  const int a0 = blockIdx.x * kTile, l0 = blockIdx.y * kTile;
  const int64_t ip = blockIdx.z;
  const int n = m.n;
  const int64_t org = patch_origin(m, ip);
  const int64_t ts = tstride(m);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  cf acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
  for (int src = 0; src < 2; ++src) {
    const cf* Mp = (src ? K : W) + ip * (int64_t)n * n;
    const cf* img = src ? z : xb;
    for (int b0 = 0; b0 < n; b0 += kKc) {
      for (int q = threadIdx.x; q < kKc * kTile; q += blockDim.x) {
        {   // matrix tile As[b][a] = W[a][b] (row-major: b contiguous)
          const int kk = q % kKc, r = q / kKc;
          const int a = a0 + r, b = b0 + kk;
          cf w = make_float2(0.f, 0.f);
          if (a < n && b < n) {
            w = Mp[(int64_t)a * n + b];
            if (m.tall) w = cconj(w);
          }
          As[kk][r] = w;
        }
        {
          int kk, r;
          if (m.tall) {
            r = q % kTile;
            kk = q / kTile;
          } else {
            kk = q % kKc;
            r = q / kKc;
          }
          const int b = b0 + kk, l = l0 + r;
          cf v = make_float2(0.f, 0.f);
          if (b < n && l < m.L) {
            v = m.tall ? img[org + patch_off(m, l) + (int64_t)b * ts]
                       : img[org + patch_off(m, b) + (int64_t)l * ts];
          }
          Bs[kk][r] = v;
        }
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < kKc; ++kk) {
        cf av[4], bv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) av[i] = As[kk][ty * 4 + i];
#pragma unroll
        for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx * 4 + j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            acc[i][j].x += av[i].x * bv[j].x - av[i].y * bv[j].y;
            acc[i][j].y += av[i].x * bv[j].y + av[i].y * bv[j].x;
          }
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int a = a0 + ty * 4 + i, l = l0 + tx * 4 + j;
      if (a >= n || l >= m.L) continue;
      const int pv = m.tall ? l : a;
      const int tt = m.tall ? a : l;
      if (direct) out[org + patch_off(m, pv) + (int64_t)tt * ts] = acc[i][j];
      else out[(ip * m.Nt + tt) * (int64_t)m.p + pv] = acc[i][j];
    }
}

// Coverage count of voxel (x, y, z) from the per-dimension covering ranges.
__device__ __forceinline__ float cover_count(const int* cover, const PatchMap& m, int64_t v) {
  const int x = (int)(v % m.Nx);
  const int y = (int)((v / m.Nx) % m.Ny);
  const int z = (int)(v / ((int64_t)m.Nx * m.Ny));
  const int* cx = cover;
  const int* cy = cover + 2 * m.Nx;
  const int* cz = cy + 2 * m.Ny;
  if (cx[2 * x] < 0 || cy[2 * y] < 0 || cz[2 * z] < 0) return 0.f;
  return (float)((cx[2 * x + 1] - cx[2 * x] + 1) * (cy[2 * y + 1] - cy[2 * y] + 1) *
                 (cz[2 * z + 1] - cz[2 * z] + 1));
}

// out = img / max(count, 1): the adjoint of patches2img's averaging, before the gather
__global__ void k_div_count(const cf* __restrict__ img, PatchMap m, const int* __restrict__ cover,
                            cf* __restrict__ out) {
  const int64_t total = (int64_t)m.Nt * m.nvox;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const float c = fmaxf(cover_count(cover, m, q % m.nvox), 1.f);
    out[q] = make_float2(img[q].x / c, img[q].y / c);
  }
}

// Scatter-add of per-patch values (the adjoint of img2patches) as a gather
// over covering patches in ascending ip; uncovered voxels get 0.
__global__ void k_patch_sum(const cf* __restrict__ P, PatchMap m, const int* __restrict__ cover,
                            cf* __restrict__ img) {
  const int64_t total = (int64_t)m.Nt * m.nvox;
  const int* cx = cover;
  const int* cy = cover + 2 * m.Nx;
  const int* cz = cy + 2 * m.Ny;
  const int* sxs = m.starts;
  const int* sys = m.starts + m.nx;
  const int* szs = m.starts + m.nx + m.ny;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = q % m.nvox;
    const int t = (int)(q / m.nvox);
    const int x = (int)(v % m.Nx);
    const int y = (int)((v / m.Nx) % m.Ny);
    const int z = (int)(v / ((int64_t)m.Nx * m.Ny));
    cf acc = make_float2(0.f, 0.f);
    if (cx[2 * x] >= 0 && cy[2 * y] >= 0 && cz[2 * z] >= 0) {
      for (int iz = cz[2 * z]; iz <= cz[2 * z + 1]; ++iz)
        for (int iy = cy[2 * y]; iy <= cy[2 * y + 1]; ++iy)
          for (int ix = cx[2 * x]; ix <= cx[2 * x + 1]; ++ix) {
            const int64_t ip = ix + (int64_t)m.nx * (iy + (int64_t)m.ny * iz);
            const int l = (x - sxs[ix]) + m.psx * ((y - sys[iy]) + m.psy * (z - szs[iz]));
            acc = cadd(acc, P[(ip * m.Nt + t) * (int64_t)m.p + l]);
          }
    }
    img[q] = acc;
  }
}

// r = Σ_k X_k − X_true;  xbar_k = r for every scale;  part[b] = Σ |r|² (FP64)
__global__ void __launch_bounds__(256) k_loss_seed(const cf* __restrict__ X, const cf* __restrict__ Xt,
                                                   int ns, int64_t E, cf* __restrict__ xbar,
                                                   double* __restrict__ part) {
  __shared__ double red[8];
  double s = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
       e += (int64_t)gridDim.x * blockDim.x) {
    cf r = X[e];
    for (int k = 1; k < ns; ++k) r = cadd(r, X[k * E + e]);
    r = csub(r, Xt[e]);
    for (int k = 0; k < ns; ++k) xbar[k * E + e] = r;
    s += (double)r.x * r.x + (double)r.y * r.y;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[w];
    part[blockIdx.x] = t;
  }
}

// w = ū + a z̄   (all scales)
__global__ void k_axpy2(const cf* __restrict__ ub, const cf* __restrict__ zb, float a, int64_t n,
                        cf* __restrict__ w) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    w[e] = make_float2(ub[e].x + a * zb[e].x, ub[e].y + a * zb[e].y);
}

// x̄_k = w_k − α h − γ z̄_k,  ū_k = −β z̄_k   (h = A'A Σ_k w_k, one image)
__global__ void k_adj_step(const cf* __restrict__ w, const cf* __restrict__ h, const cf* __restrict__ zb,
                           float alpha, float beta, float gamma, int ns, int64_t E, cf* __restrict__ xb,
                           cf* __restrict__ ub) {
  const int64_t n = (int64_t)ns * E;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const cf hv = h[e % E], zv = zb[e], wv = w[e];
    xb[e] = make_float2(wv.x - alpha * hv.x - gamma * zv.x, wv.y - alpha * hv.y - gamma * zv.y);
    ub[e] = make_float2(-beta * zv.x, -beta * zv.y);
  }
}

}  // namespace

int xgram_launch(const cf* imgO, const cf* imgM, const PatchMap& m, int64_t np, cf* out, cf* part,
                 int nsplit, cudaStream_t st) {
  const int T = (m.n + kTile - 1) / kTile;
  const int lchunk = (nsplit > 1) ? ((m.L + nsplit - 1) / nsplit + kKc - 1) / kKc * kKc : m.L;
  k_xgram<<<dim3(T * T, (unsigned)np, nsplit), 256, 0, st>>>(imgO, imgM, m, nsplit > 1 ? part : out,
                                                             nsplit, lchunk);
  if (nsplit > 1) k_split_sum<<<kRedBlocks, 256, 0, st>>>(part, out, nsplit, np * m.n * (int64_t)m.n);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int bgemm_launch(int opa, int opb, const cf* A, const cf* B, cf* C, int n, int64_t np, cudaStream_t st) {
  const int T = (n + kTile - 1) / kTile;
  const dim3 grid(T * T, (unsigned)np);
  if (opa == 0 && opb == 0) k_bgemm<0, 0><<<grid, 256, 0, st>>>(A, B, C, n);
  else if (opa == 1 && opb == 0) k_bgemm<1, 0><<<grid, 256, 0, st>>>(A, B, C, n);
  else if (opa == 0 && opb == 1) k_bgemm<0, 1><<<grid, 256, 0, st>>>(A, B, C, n);
  else k_bgemm<1, 1><<<grid, 256, 0, st>>>(A, B, C, n);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int divdiff_launch(const cf* D, const double* lam, const cf* V, double beta, int n, int64_t np, cf* E,
                   cf* T3, double* bbar, cudaStream_t st) {
  k_divdiff<<<(unsigned)np, 256, 0, st>>>(D, lam, V, beta, n, E, T3, bbar);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int vjp_rebuild_launch(const cf* xb, const cf* z, const cf* W, const cf* K, const PatchMap& m,
                       int64_t np, cf* out, int direct, cudaStream_t st) {
  k_vjp_rebuild<<<dim3((m.n + kTile - 1) / kTile, (m.L + kTile - 1) / kTile, (unsigned)np), 256, 0,
                  st>>>(xb, z, W, K, m, out, direct);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int div_count_launch(const cf* img, const PatchMap& m, const int* cover, cf* out, cudaStream_t st) {
  k_div_count<<<1184, 256, 0, st>>>(img, m, cover, out);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int patch_sum_launch(const cf* P, const PatchMap& m, const int* cover, cf* img, cudaStream_t st) {
  k_patch_sum<<<1184, 256, 0, st>>>(P, m, cover, img);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

// ---------------------------------------------------------------------------
// Unrolled-POGM gradient
// ---------------------------------------------------------------------------
int set_lambdas(Ctx* c, const double* lam) {
  for (int k = 0; k < c->Ns; ++k) {
    if (!(lam[k] >= 0.0) || !std::isfinite(lam[k]))
      return fail(MSLR_ERR_ARG, "lambdas must be finite and non-negative");
  }
  for (int k = 0; k < c->Ns; ++k) c->lambdas[k] = lam[k];
  // the captured iteration holds the thresholds' scale factors as launch arguments
  if (c->gexec) {
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
    c->gX = nullptr;
  }
  return MSLR_OK;
}

int pogm_grad(Ctx* c, const cf* Xtrue, int niter, double L, double cutoff, double bsig, cf* X,
              double* loss, double* grad, uint8_t* restarts_h, cudaStream_t st) {
  int rc;
  const int Ns = c->Ns;
  const int64_t E = (int64_t)c->Nt * c->nvox;
  const size_t slot = (size_t)Ns * E;
  if (niter > c->grad_ckpt_cap) {
    if (c->d_ckpt) cudaFree(c->d_ckpt);
    c->d_ckpt = nullptr;
    c->grad_ckpt_cap = 0;
    if ((rc = dalloc(c, (void**)&c->d_ckpt, (size_t)niter * slot * sizeof(cf)))) return rc;
    c->grad_ckpt_cap = niter;
  }
  if (!c->d_gbuf) {
    // x̄, ū, z̄, w (Ns slots each), h, temporary image, loss partials
    if ((rc = dalloc(c, (void**)&c->d_gbuf, (4 * slot + 2 * (size_t)E) * sizeof(cf) +
                                                 kRedBlocks * sizeof(double))))
      return rc;
  }
  if ((rc = svst_vjp_setup(c))) return rc;
  cf* xb = c->d_gbuf;
  cf* ub = xb + slot;
  cf* zb = ub + slot;
  cf* wv = zb + slot;
  cf* h = wv + slot;
  cf* tmp = h + E;
  double* part = reinterpret_cast<double*>(tmp + E);

  // forward, keeping z_i and the momentum scalars of every iteration
  if ((rc = init_x0(c, X, st))) return rc;
  if ((rc = pogm_begin(c, X, niter, L, cutoff, bsig, st))) return rc;
  std::vector<PogmState> sc(niter);
  for (int i = 0; i < niter; ++i) {
    if ((rc = pogm_step(c, X, st))) return rc;
    MSLR_CUDA_TRY(cudaMemcpyAsync(c->d_ckpt + (size_t)i * slot, c->d_Z, slot * sizeof(cf),
                                  cudaMemcpyDeviceToDevice, st));
    MSLR_CUDA_TRY(cudaMemcpyAsync(&sc[i], c->d_state, sizeof(PogmState), cudaMemcpyDeviceToHost, st));
  }
  if (restarts_h)
    MSLR_CUDA_TRY(cudaMemcpyAsync(restarts_h, c->d_restarts, (size_t)niter + 1, cudaMemcpyDeviceToHost, st));

  // loss and x̄_N
  k_loss_seed<<<kRedBlocks, 256, 0, st>>>(X, Xtrue, Ns, E, xb, part);
  MSLR_CUDA_TRY(cudaGetLastError());
  std::vector<double> hp(kRedBlocks);
  MSLR_CUDA_TRY(cudaMemcpyAsync(hp.data(), part, kRedBlocks * sizeof(double), cudaMemcpyDeviceToHost, st));
  MSLR_CUDA_TRY(cudaMemsetAsync(ub, 0, slot * sizeof(cf), st));
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  double l2 = 0.0;
  for (double v : hp) l2 += v;
  *loss = 0.5 * l2;
  for (int k = 0; k < Ns; ++k) grad[k] = 0.0;

  for (int i = niter - 1; i >= 0; --i) {
    const PogmState& s = sc[i];
    const cf* z = c->d_ckpt + (size_t)i * slot;
    for (int k = 0; k < Ns; ++k) {
      const double thr = s.zeta * c->lambdas[k];
      double bb = 0.0;
      if ((rc = svst_vjp_scale(c, k, z + k * E, xb + k * E, thr, zb + k * E, tmp, &bb, st))) return rc;
      grad[k] += thr * bb;
    }
    k_axpy2<<<1184, 256, 0, st>>>(ub, zb, (float)(1.0 + s.beta + s.gamma), (int64_t)slot, wv);
    MSLR_CUDA_TRY(cudaGetLastError());
    if ((rc = normal_op(c, wv, Ns, E, h, false, st))) return rc;
    k_adj_step<<<1184, 256, 0, st>>>(wv, h, zb, (float)s.alpha, (float)s.beta, (float)s.gamma, Ns, E,
                                      xb, ub);
    MSLR_CUDA_TRY(cudaGetLastError());
  }
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  return MSLR_OK;
}

}  // namespace mslr
