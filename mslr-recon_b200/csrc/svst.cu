// svst.cu — batched patch SVST on sm_100a (plain FP32 SIMT form).
//
// Reference: img2patches / patches2img (src/recon.jl:53-126), SVST
// (src/recon.jl:183-211; src/sense_gpu.jl:122-128) and patchSVST
// (src/recon.jl:251-269; src/sense_gpu.jl:138-160).
//
// For a patch matrix P (p × Nt) let n = min(p, Nt) and M be the n × L matrix
//   M = Pᴴ (p ≥ Nt, "tall")   or   M = P (p < Nt, "wide"),
// so that G = M Mᴴ is the smaller Gram matrix.  With G = V diag(λ) Vᴴ and
// σ = √λ, SVST(P) = U diag(max(σ − β, 0)) Vᴴ equals
//   W = V diag(h) Vᴴ,  h = max(σ − β, 0)/σ,   M_out = W M,
// and P_out = M_outᴴ (tall) or M_out (wide).  Zero patches give G = 0, no
// eigenvalue above β², W = 0 and a zero output: the reference's zero-norm
// skip (src/recon.jl:185) falls out without a special case.
//
// Per patch (one CTA):
//   1. Householder tridiagonalisation of G (FP32, FP64 reductions),
//   2. eigenvalues above β² by Sturm bisection on the real tridiagonal (FP64),
//   3. eigenvectors by twisted factorisation (FP64), MGS within tight clusters,
//   4. back-transformation by the Householder reflectors,
//   5. W = V diag(h) Vᴴ.
// Patches never see a host loop: every stage is one launch over all patches
// of a scale.  Overlapping or gapped patch grids are recombined by a gather
// over covering patches in ascending ip order with the Float32 coverage
// count, clamped to 1 (src/recon.jl:113-124).
#include <algorithm>
#include <cmath>
#include <mutex>

#include "internal.h"

namespace mslr {

namespace {

constexpr int kEigThreads = 256;
constexpr int kTile = 64;
constexpr int kKc = 16;

// Device-side addressing of patch elements.  Element (l, t) of patch ip —
// l the in-patch voxel (x fastest), t the frame — lives at
//   image mode: origin(ip) + lx + Nx (ly + Ny lz) + t·nvox
//   batch mode: ip·mstride + l + t·m        (column-major m × Nt matrices)
struct PatchMap {
  int Nx, Ny, Nz;
  int64_t nvox;
  int Nt;
  int psx, psy, psz;
  int nx, ny, nz;     // patches per dim
  const int* starts;  // nx x-starts, ny y-starts, nz z-starts
  int p, n, L;
  int tall;
  int batch;
  int64_t mstride;
};

__device__ __forceinline__ int64_t patch_origin(const PatchMap& m, int64_t ip) {
  if (m.batch) return ip * m.mstride;
  const int ix = (int)(ip % m.nx);
  const int iy = (int)((ip / m.nx) % m.ny);
  const int iz = (int)(ip / ((int64_t)m.nx * m.ny));
  const int sx = m.starts[ix], sy = m.starts[m.nx + iy], sz = m.starts[m.nx + m.ny + iz];
  return sx + (int64_t)m.Nx * (sy + (int64_t)m.Ny * sz);
}

__device__ __forceinline__ int64_t patch_off(const PatchMap& m, int l) {
  if (m.batch) return l;
  const int lx = l % m.psx;
  const int r = l / m.psx;
  const int ly = r % m.psy;
  const int lz = r / m.psy;
  return lx + (int64_t)m.Nx * (ly + (int64_t)m.Ny * lz);
}

__device__ __forceinline__ int64_t tstride(const PatchMap& m) { return m.batch ? (int64_t)m.p : m.nvox; }

// M[a][l] of patch with origin `org`
__device__ __forceinline__ cf m_elem(const PatchMap& m, const cf* __restrict__ img, int64_t org,
                                     int a, int l) {
  if (m.tall) {
    const cf v = img[org + patch_off(m, l) + (int64_t)a * tstride(m)];
    return cconj(v);
  }
  return img[org + patch_off(m, a) + (int64_t)l * tstride(m)];
}

// ---------------------------------------------------------------------------
// Gram: G[a][b] = Σ_l M[a][l] conj(M[b][l]) on lower-triangle 64×64 tiles.
// grid (ntri, Np, nsplit).  Output column-major: G[b*n + a].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_gram(const cf* __restrict__ img, PatchMap m,
                                              cf* __restrict__ out, int nsplit, int lchunk) {
  __shared__ cf As[kKc][kTile + 1];
  __shared__ cf Bs[kKc][kTile + 1];
  // tile pair from the linear lower-triangle index
  int t = blockIdx.x, ta = 0;
  while (t > ta) {
    t -= ta + 1;
    ++ta;
  }
  const int tb = t;
  const int64_t ip = blockIdx.y;
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
    // load: 1024 elements each for A and B; kk fastest for tall (voxel-contiguous)
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
        if (a0 + r < m.n) va = m_elem(m, img, org, a0 + r, l);
        if (b0 + r < m.n) vb = m_elem(m, img, org, b0 + r, l);
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
          // av * conj(bv)
          acc[i][j].x += av[i].x * bv[j].x + av[i].y * bv[j].y;
          acc[i][j].y += av[i].y * bv[j].x - av[i].x * bv[j].y;
        }
    }
    __syncthreads();
  }
  const int n = m.n;
  cf* G = out + ((nsplit > 1) ? (int64_t)split * n * n : ip * (int64_t)n * n);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int a = a0 + ty * 4 + i, b = b0 + tx * 4 + j;
      if (a < n && b < n) {
        G[(int64_t)b * n + a] = acc[i][j];
        if (ta != tb) G[(int64_t)a * n + b] = cconj(acc[i][j]);
      }
    }
}

__global__ void k_gram_reduce(const cf* __restrict__ part, cf* __restrict__ G, int nsplit,
                              int64_t nn) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nn;
       e += (int64_t)gridDim.x * blockDim.x) {
    cf s = part[e];
    for (int q = 1; q < nsplit; ++q) s = cadd(s, part[q * nn + e]);
    G[e] = s;
  }
}

// ---------------------------------------------------------------------------
// Per-patch eigen stage.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// block-wide double sum; result broadcast to all threads
__device__ double block_sum_all(double v, double* sh) {
  v = warp_sum_d(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];
  return r;
}

// number of eigenvalues of the symmetric tridiagonal (d, e) strictly below x
__device__ int sturm_less(const double* d, const double* e, int n, double x, double pivmin) {
  int cnt = 0;
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  if (q < 0) ++cnt;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - (e[i - 1] * e[i - 1]) / q;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0) ++cnt;
  }
  return cnt;
}

struct EigArgs {
  int n;
  cf* gram;          // np*n*n
  void* zv;          // np*n*n × 8 bytes
  double* aux;       // np*n*n
  double* vecs;      // np*6*n
  int* rank;         // np
  const double* thr; // device threshold(s)
  int thr_per_patch;
  double lam;
};

__global__ void __launch_bounds__(kEigThreads) k_eig(EigArgs g) {
  extern __shared__ unsigned char smraw[];
  const int n = g.n;
  const int64_t ip = blockIdx.x;
  cf* A = g.gram + ip * (int64_t)n * n;
  double* Z = reinterpret_cast<double*>(g.zv) + ip * (int64_t)n * n;
  cf* V = reinterpret_cast<cf*>(g.zv) + ip * (int64_t)n * n;
  double* AUX = g.aux + ip * (int64_t)n * n;
  double* vec = g.vecs + ip * (int64_t)6 * n;
  double* d = vec;              // n
  double* e = vec + n;          // n
  double* taur = vec + 2 * n;   // n
  double* taui = vec + 3 * n;   // n
  double* lamv = vec + 4 * n;   // n
  double* hv = vec + 5 * n;     // n
  cf* sv = reinterpret_cast<cf*>(smraw);   // n
  cf* sy = sv + n;                          // n (y then w)
  double* red = reinterpret_cast<double*>(sy + n);  // 32
  __shared__ double s_bc[8];
  __shared__ int s_r;
  const int tid = threadIdx.x, nt = blockDim.x;

  const double beta = g.thr[g.thr_per_patch ? ip : 0] * g.lam;
  const double thr2 = beta * beta;

  // ---- 1. Householder tridiagonalisation, A ← Hᴴ A H per step --------------
  for (int k = 0; k < n - 1; ++k) {
    const int m = n - k - 1;
    cf* colk = A + (int64_t)k * n;
    double xn = 0.0;
    for (int i = k + 2 + tid; i < n; i += nt) {
      const cf v = colk[i];
      xn += (double)v.x * v.x + (double)v.y * v.y;
    }
    xn = block_sum_all(xn, red);
    if (tid == 0) {
      const cf al = colk[k + 1];
      const double ar = al.x, ai = al.y;
      double bt, tr, ti, sr, si;
      if (xn == 0.0 && ai == 0.0) {
        bt = ar;
        tr = ti = 0.0;
        sr = 1.0;
        si = 0.0;
      } else {
        bt = -copysign(sqrt(ar * ar + ai * ai + xn), ar);
        tr = (bt - ar) / bt;
        ti = -ai / bt;
        const double zr = ar - bt, zi = ai;
        const double den = zr * zr + zi * zi;
        sr = zr / den;
        si = -zi / den;
      }
      d[k] = (double)colk[k].x;
      e[k] = bt;
      taur[k] = tr;
      taui[k] = ti;
      s_bc[0] = tr;
      s_bc[1] = ti;
      s_bc[2] = sr;
      s_bc[3] = si;
    }
    __syncthreads();
    const float tr = (float)s_bc[0], ti = (float)s_bc[1];
    const cf scal = make_float2((float)s_bc[2], (float)s_bc[3]);
    for (int i = tid; i < m; i += nt) {
      cf v;
      if (i == 0) {
        v = make_float2(1.f, 0.f);
      } else {
        v = cmul(colk[k + 1 + i], scal);
        colk[k + 1 + i] = v;   // Householder vector kept below the subdiagonal
      }
      sv[i] = v;
    }
    __syncthreads();
    if (tr == 0.f && ti == 0.f) continue;
    const cf tau = make_float2(tr, ti);
    // y = A22 v
    cf* A22 = A + (int64_t)(k + 1) * n + (k + 1);
    for (int i = tid; i < m; i += nt) {
      float yr = 0.f, yi = 0.f;
      for (int j = 0; j < m; ++j) {
        const cf a = A22[(int64_t)j * n + i];
        const cf v = sv[j];
        yr += a.x * v.x - a.y * v.y;
        yi += a.x * v.y + a.y * v.x;
      }
      sy[i] = make_float2(yr, yi);
    }
    __syncthreads();
    double vy = 0.0;   // Re(vᴴ y)
    for (int i = tid; i < m; i += nt) vy += (double)sv[i].x * sy[i].x + (double)sv[i].y * sy[i].y;
    vy = block_sum_all(vy, red);
    const float cst = (float)(0.5 * ((double)tr * tr + (double)ti * ti) * vy);
    for (int i = tid; i < m; i += nt) {
      const cf w = csub(cmul(tau, sy[i]), cscale(sv[i], cst));
      sy[i] = w;
    }
    __syncthreads();
    // A22 −= w vᴴ + v wᴴ
    for (int i = tid; i < m; i += nt) {
      const cf wi = sy[i], vi = sv[i];
      for (int j = 0; j < m; ++j) {
        const cf vj = sv[j], wj = sy[j];
        cf a = A22[(int64_t)j * n + i];
        a = csub(a, cmul(wi, cconj(vj)));
        a = csub(a, cmul(vi, cconj(wj)));
        A22[(int64_t)j * n + i] = a;
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    d[n - 1] = (double)A[(int64_t)(n - 1) * n + (n - 1)].x;
    if (n >= 1) e[n - 1] = 0.0;
  }
  __syncthreads();

  // ---- 2. eigenvalues above β² --------------------------------------------
  if (tid == 0) {
    double gl = d[0], gu = d[0], emax2 = 0.0;
    for (int i = 0; i < n; ++i) {
      const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
      gl = fmin(gl, d[i] - r);
      gu = fmax(gu, d[i] + r);
      if (i < n - 1) emax2 = fmax(emax2, e[i] * e[i]);
    }
    const double tnorm = fmax(fabs(gl), fabs(gu));
    const double pivmin = fmax(2.2250738585072014e-308 * fmax(emax2, 1.0), 1e-300);
    gl -= 2.0 * 2.220446049250313e-16 * tnorm * n + pivmin;
    gu += 2.0 * 2.220446049250313e-16 * tnorm * n + pivmin;
    s_bc[4] = gl;
    s_bc[5] = gu;
    s_bc[6] = pivmin;
    s_bc[7] = tnorm;
    const int below = sturm_less(d, e, n, thr2, pivmin);
    s_r = (thr2 >= gu) ? 0 : n - below;
  }
  __syncthreads();
  const int r = s_r;
  const double gl = s_bc[4], gu = s_bc[5], pivmin = s_bc[6], tnorm = s_bc[7];
  if (tid == 0) g.rank[ip] = r;
  for (int i = tid; i < r; i += nt) {
    const int kth = n - 1 - i;   // kth smallest
    double lo = gl, hi = gu;
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (hi - lo <= 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)) + pivmin || mid == lo ||
          mid == hi)
        break;
      if (sturm_less(d, e, n, mid, pivmin) > kth) hi = mid;
      else lo = mid;
    }
    const double lm = 0.5 * (lo + hi);
    lamv[i] = lm;
    const double sg = sqrt(fmax(lm, 0.0));
    hv[i] = (sg > beta && sg > 0.0) ? (sg - beta) / sg : 0.0;
  }
  __syncthreads();
  if (r == 0) {
    for (int64_t q = tid; q < (int64_t)n * n; q += nt) A[q] = make_float2(0.f, 0.f);
    return;
  }

  // ---- 3. eigenvectors of T by twisted factorisation -------------------------
  for (int i = tid; i < r; i += nt) {
    const double lm = lamv[i];
    double* z = Z + (int64_t)i * n;     // holds D+ then z
    double* dm = AUX + (int64_t)i * n;  // D−
    z[0] = d[0] - lm;
    if (fabs(z[0]) < pivmin) z[0] = -pivmin;
    for (int j = 0; j + 1 < n; ++j) {
      double q = d[j + 1] - lm - e[j] * e[j] / z[j];
      if (fabs(q) < pivmin) q = -pivmin;
      z[j + 1] = q;
    }
    dm[n - 1] = d[n - 1] - lm;
    if (fabs(dm[n - 1]) < pivmin) dm[n - 1] = -pivmin;
    for (int j = n - 2; j >= 0; --j) {
      double q = d[j] - lm - e[j] * e[j] / dm[j + 1];
      if (fabs(q) < pivmin) q = -pivmin;
      dm[j] = q;
    }
    int kb = 0;
    double gb = INFINITY;
    for (int j = 0; j < n; ++j) {
      const double gm = fabs(z[j] + dm[j] - (d[j] - lm));
      if (gm < gb) {
        gb = gm;
        kb = j;
      }
    }
    // z_kb = 1; upward with D+, downward with D−
    double nrm = 1.0;
    double zprev = 1.0;
    for (int j = kb - 1; j >= 0; --j) {
      const double zj = -e[j] * zprev / z[j];
      z[j] = zj;
      zprev = zj;
      nrm += zj * zj;
    }
    z[kb] = 1.0;
    zprev = 1.0;
    for (int j = kb + 1; j < n; ++j) {
      const double zj = -e[j - 1] * zprev / dm[j];
      z[j] = zj;
      zprev = zj;
      nrm += zj * zj;
    }
    const double inv = 1.0 / sqrt(nrm);
    for (int j = 0; j < n; ++j) z[j] *= inv;
  }
  __syncthreads();
  // tight clusters: modified Gram–Schmidt (one thread; clusters are rare)
  if (tid == 0) {
    const double ctol = 1e-10 * fmax(tnorm, 1e-300);
    int s = 0;
    while (s < r) {
      int t = s + 1;
      while (t < r && lamv[t - 1] - lamv[t] <= ctol) ++t;
      if (t - s > 1) {
        for (int q = s; q < t; ++q) {
          double* zq = Z + (int64_t)q * n;
          for (int attempt = 0; attempt < 4; ++attempt) {
            for (int p2 = s; p2 < q; ++p2) {
              const double* zp = Z + (int64_t)p2 * n;
              double dot = 0.0;
              for (int j = 0; j < n; ++j) dot += zp[j] * zq[j];
              for (int j = 0; j < n; ++j) zq[j] -= dot * zp[j];
            }
            double nr = 0.0;
            for (int j = 0; j < n; ++j) nr += zq[j] * zq[j];
            nr = sqrt(nr);
            if (nr > 0.1) {
              for (int j = 0; j < n; ++j) zq[j] /= nr;
              break;
            }
            // collapsed: restart from a deterministic unit vector and retry
            for (int j = 0; j < n; ++j) zq[j] = 0.0;
            zq[(q + attempt * 7919) % n] = 1.0;
          }
        }
      }
      s = t;
    }
  }
  __syncthreads();

  // ---- 4. back-transformation V = H_0 … H_{n-2} Z ----------------------------
  for (int i = tid; i < r; i += nt) {
    double* z = Z + (int64_t)i * n;
    cf* vcol = V + (int64_t)i * n;
    for (int j = 0; j < n; ++j) {
      const double zj = z[j];
      vcol[j] = make_float2((float)zj, 0.f);
    }
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
  for (int k = n - 2; k >= 0; --k) {
    const float tr = (float)taur[k], ti = (float)taui[k];
    if (tr == 0.f && ti == 0.f) continue;
    const int m = n - k - 1;
    const cf* colk = A + (int64_t)k * n;
    for (int i = tid; i < m; i += nt) sv[i] = (i == 0) ? make_float2(1.f, 0.f) : colk[k + 1 + i];
    __syncthreads();
    const cf tau = make_float2(tr, ti);
    for (int j = warp; j < r; j += nw) {
      cf* vc = V + (int64_t)j * n + (k + 1);
      float sr = 0.f, si = 0.f;
      for (int i = lane; i < m; i += 32) {
        const cf a = sv[i], b = vc[i];   // conj(a)·b
        sr += a.x * b.x + a.y * b.y;
        si += a.x * b.y - a.y * b.x;
      }
      for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
      }
      const cf ts = cmul(tau, make_float2(sr, si));
      for (int i = lane; i < m; i += 32) vc[i] = csub(vc[i], cmul(sv[i], ts));
    }
    __syncthreads();
  }

  // ---- 5. W = V diag(h) Vᴴ into A ------------------------------------------
  for (int64_t q = tid; q < (int64_t)n * n; q += nt) {
    const int a = (int)(q % n), b = (int)(q / n);
    float wr = 0.f, wi = 0.f;
    for (int i = 0; i < r; ++i) {
      const float h = (float)hv[i];
      const cf va = V[(int64_t)i * n + a], vb = V[(int64_t)i * n + b];
      // h · va · conj(vb)
      wr += h * (va.x * vb.x + va.y * vb.y);
      wi += h * (va.y * vb.x - va.x * vb.y);
    }
    A[(int64_t)b * n + a] = make_float2(wr, wi);
  }
}

// ---------------------------------------------------------------------------
// Rebuild: M_out = W M.  tall: out[t=a][vox_l] = Σ_b conj(W[a][b]) img[b][vox_l]
//                       wide: out[t=l][vox_a] = Σ_b W[a][b] img[l][vox_b]
// grid (ceil(n/64), ceil(L/64), Np).  Writes the image directly when the
// patch grid is an exact partition, else the per-patch buffer (p, Nt, Np).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_rebuild(const cf* __restrict__ img, const cf* __restrict__ W,
                                                 PatchMap m, cf* __restrict__ out, int direct) {
  __shared__ cf As[kKc][kTile + 1];   // W[a][b]
  __shared__ cf Bs[kKc][kTile + 1];   // input values for (b, l)
  const int a0 = blockIdx.x * kTile, l0 = blockIdx.y * kTile;
  const int64_t ip = blockIdx.z;
  const int n = m.n;
  const cf* Wp = W + ip * (int64_t)n * n;
  const int64_t org = patch_origin(m, ip);
  const int64_t ts = tstride(m);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  cf acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
  for (int b0 = 0; b0 < n; b0 += kKc) {
    for (int q = threadIdx.x; q < kKc * kTile; q += blockDim.x) {
      // W tile: a fastest (column-major W[b*n + a])
      {
        const int r = q % kTile, kk = q / kTile;
        const int a = a0 + r, b = b0 + kk;
        cf w = make_float2(0.f, 0.f);
        if (a < n && b < n) {
          w = Wp[(int64_t)b * n + a];
          if (m.tall) w = cconj(w);
        }
        As[kk][r] = w;
      }
      // input tile
      {
        int kk, r;
        if (m.tall) {   // img[b][vox_l]: l contiguous
          r = q % kTile;
          kk = q / kTile;
        } else {        // img[l][vox_b]: b contiguous
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
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int a = a0 + ty * 4 + i, l = l0 + tx * 4 + j;
      if (a >= n || l >= m.L) continue;
      // element (voxel, frame) of the patch
      const int pv = m.tall ? l : a;
      const int tt = m.tall ? a : l;
      if (direct) out[org + patch_off(m, pv) + (int64_t)tt * ts] = acc[i][j];
      else out[(ip * m.Nt + tt) * (int64_t)m.p + pv] = acc[i][j];
    }
}

// img2patches: P[(ip*Nt + t)*p + l] = img[t][vox(ip, l)]
__global__ void k_img2patches(const cf* __restrict__ img, PatchMap m, cf* __restrict__ P,
                              int64_t total) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int l = (int)(q % m.p);
    const int64_t r = q / m.p;
    const int t = (int)(r % m.Nt);
    const int64_t ip = r / m.Nt;
    P[q] = img[patch_origin(m, ip) + patch_off(m, l) + (int64_t)t * m.nvox];
  }
}

// Gather recombine (patches2img): for voxel v and frame t, Σ over covering
// patches in ascending ip of P[(ip*Nt + t)*p + l(v, ip)], divided by
// max(count, 1).  cover: per dim 2*N[d] ints (lo, hi) of covering indices.
__global__ void k_recombine(const cf* __restrict__ P, PatchMap m, const int* __restrict__ cover,
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
    const int xl = cx[2 * x], xh = cx[2 * x + 1];
    const int yl = cy[2 * y], yh = cy[2 * y + 1];
    const int zl = cz[2 * z], zh = cz[2 * z + 1];
    cf acc = make_float2(0.f, 0.f);
    float cnt = 0.f;
    if (xl >= 0 && yl >= 0 && zl >= 0) {
      for (int iz = zl; iz <= zh; ++iz)
        for (int iy = yl; iy <= yh; ++iy)
          for (int ix = xl; ix <= xh; ++ix) {
            const int64_t ip = ix + (int64_t)m.nx * (iy + (int64_t)m.ny * iz);
            const int l = (x - sxs[ix]) + m.psx * ((y - sys[iy]) + m.psy * (z - szs[iz]));
            acc = cadd(acc, P[(ip * m.Nt + t) * (int64_t)m.p + l]);
            cnt += 1.f;
          }
    }
    cnt = fmaxf(cnt, 1.f);
    img[q] = make_float2(acc.x / cnt, acc.y / cnt);
  }
}

__global__ void k_zero(cf* p, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    p[q] = make_float2(0.f, 0.f);
}

PatchMap map_of(const ScaleGeom& g, const int N[3], int Nt, int64_t nvox) {
  PatchMap m;
  m.Nx = N[0];
  m.Ny = N[1];
  m.Nz = N[2];
  m.nvox = nvox;
  m.Nt = Nt;
  m.psx = g.ps[0];
  m.psy = g.ps[1];
  m.psz = g.ps[2];
  m.nx = g.nsteps[0] + 1;
  m.ny = g.nsteps[1] + 1;
  m.nz = g.nsteps[2] + 1;
  m.starts = g.d_starts;
  m.p = g.p;
  m.n = g.n;
  m.L = g.L;
  m.tall = g.tall ? 1 : 0;
  m.batch = 0;
  m.mstride = 0;
  return m;
}

size_t eig_smem(int n) { return (size_t)2 * n * sizeof(cf) + 32 * sizeof(double); }

struct WorkPtrs {
  cf* gram;
  void* zv;
  double* aux;
  double* vecs;
  int* rank;
  cf* part;
};

// Gram → eig → (rebuild into out or pbuf) for all patches described by m.
int svst_core(const cf* in, const PatchMap& m, int64_t np, const WorkPtrs& w, int nsplit,
              const double* thr, int thr_per_patch, double lam, cf* out, int direct,
              cudaStream_t st, uint64_t* launches) {
  if (launches) *launches += (nsplit > 1 ? 4 : 3);
  const int n = m.n;
  const int T = (n + kTile - 1) / kTile;
  const int ntri = T * (T + 1) / 2;
  if (nsplit > 1) {
    const int lchunk = ((m.L + nsplit - 1) / nsplit + kKc - 1) / kKc * kKc;
    k_gram<<<dim3(ntri, (unsigned)np, nsplit), 256, 0, st>>>(in, m, w.part, nsplit, lchunk);
    k_gram_reduce<<<592, 256, 0, st>>>(w.part, w.gram, nsplit, (int64_t)n * n);
  } else {
    k_gram<<<dim3(ntri, (unsigned)np, 1), 256, 0, st>>>(in, m, w.gram, 1, m.L);
  }
  MSLR_CUDA_TRY(cudaGetLastError());
  EigArgs ea;
  ea.n = n;
  ea.gram = w.gram;
  ea.zv = w.zv;
  ea.aux = w.aux;
  ea.vecs = w.vecs;
  ea.rank = w.rank;
  ea.thr = thr;
  ea.thr_per_patch = thr_per_patch;
  ea.lam = lam;
  k_eig<<<(unsigned)np, kEigThreads, eig_smem(n), st>>>(ea);
  MSLR_CUDA_TRY(cudaGetLastError());
  k_rebuild<<<dim3((n + kTile - 1) / kTile, (m.L + kTile - 1) / kTile, (unsigned)np), 256, 0, st>>>(
      in, w.gram, m, out, direct);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int choose_split(int64_t np, int n, int L) {
  const int T = (n + kTile - 1) / kTile;
  const int64_t ctas = (int64_t)T * (T + 1) / 2 * np;
  if (ctas >= 592) return 1;
  int s = (int)std::min<int64_t>((592 + ctas - 1) / ctas, std::max(1, L / 1024));
  return std::max(1, s);
}

}  // namespace

// ---------------------------------------------------------------------------
// geometry (host)
// ---------------------------------------------------------------------------
int geom_build(const int N[3], int Nt, const int ps_in[3], const int ss_in[3], ScaleGeom* g) {
  int64_t Np = 1;
  g->h_starts.clear();
  bool partition = true;
  for (int d = 0; d < 3; ++d) {
    if (ps_in[d] <= 0 || ss_in[d] <= 0)
      return fail(MSLR_ERR_ARG, "patch sizes and strides must be positive");
    g->ps[d] = std::min(ps_in[d], N[d]);
    g->ss[d] = ss_in[d];
    const int num = N[d] - g->ps[d];
    g->nsteps[d] = (num + g->ss[d] - 1) / g->ss[d];   // cld for num >= 0
    Np *= (g->nsteps[d] + 1);
    int prev = -1;
    for (int i = 0; i <= g->nsteps[d]; ++i) {
      const int s = std::min(i * g->ss[d], N[d] - g->ps[d]);
      g->h_starts.push_back(s);
      if (i == 0 && s != 0) partition = false;
      if (i > 0 && s - prev != g->ps[d]) partition = false;
      prev = s;
    }
    if (prev + g->ps[d] != N[d]) partition = false;
  }
  g->Np = Np;
  g->p = g->ps[0] * g->ps[1] * g->ps[2];
  g->n = std::min(g->p, Nt);
  g->L = std::max(g->p, Nt);
  g->tall = g->p >= Nt;
  g->partition = partition;
  g->global = (Np == 1 && g->ps[0] == N[0] && g->ps[1] == N[1] && g->ps[2] == N[2]);
  g->d_starts = nullptr;
  g->d_cover = nullptr;
  return MSLR_OK;
}

int geom_upload(ScaleGeom* g, const int N[3]) {
  std::vector<int> cover;
  size_t off = 0;
  for (int d = 0; d < 3; ++d) {
    const int cnt = g->nsteps[d] + 1;
    for (int c = 0; c < N[d]; ++c) {
      int lo = -1, hi = -1;
      for (int i = 0; i < cnt; ++i) {
        const int s = g->h_starts[off + i];
        if (s <= c && c < s + g->ps[d]) {
          if (lo < 0) lo = i;
          hi = i;
        }
      }
      cover.push_back(lo);
      cover.push_back(hi);
    }
    off += cnt;
  }
  MSLR_CUDA_TRY(cudaMalloc((void**)&g->d_starts, g->h_starts.size() * sizeof(int)));
  MSLR_CUDA_TRY(cudaMemcpy(g->d_starts, g->h_starts.data(), g->h_starts.size() * sizeof(int),
                           cudaMemcpyHostToDevice));
  MSLR_CUDA_TRY(cudaMalloc((void**)&g->d_cover, cover.size() * sizeof(int)));
  MSLR_CUDA_TRY(cudaMemcpy(g->d_cover, cover.data(), cover.size() * sizeof(int),
                           cudaMemcpyHostToDevice));
  return MSLR_OK;
}

void geom_free(ScaleGeom* g) {
  if (g->d_starts) cudaFree(g->d_starts);
  if (g->d_cover) cudaFree(g->d_cover);
  g->d_starts = nullptr;
  g->d_cover = nullptr;
}

static size_t eig_work_bytes(int64_t np, int n, int nsplit) {
  const size_t nn = (size_t)n * n;
  return np * nn * sizeof(cf) * 2 + np * nn * sizeof(double) + np * 6 * (size_t)n * sizeof(double) +
         np * sizeof(int) + (nsplit > 1 ? (size_t)nsplit * nn * sizeof(cf) : 0) + 6 * 256;
}

static WorkPtrs carve(void* base, int64_t np, int n, int nsplit) {
  const size_t nn = (size_t)n * n;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  unsigned char* p = reinterpret_cast<unsigned char*>(base);
  WorkPtrs w;
  w.gram = reinterpret_cast<cf*>(p);
  p += al(np * nn * sizeof(cf));
  w.zv = p;
  p += al(np * nn * sizeof(cf));
  w.aux = reinterpret_cast<double*>(p);
  p += al(np * nn * sizeof(double));
  w.vecs = reinterpret_cast<double*>(p);
  p += al(np * 6 * (size_t)n * sizeof(double));
  w.rank = reinterpret_cast<int*>(p);
  p += al(np * sizeof(int));
  w.part = nsplit > 1 ? reinterpret_cast<cf*>(p) : nullptr;
  return w;
}

int svst_setup(Ctx* c) {
  size_t need = 0, pbuf = 0;
  for (auto& g : c->scales) {
    const int nsplit = choose_split(g.Np, g.n, g.L);
    need = std::max(need, eig_work_bytes(g.Np, g.n, nsplit));
    if (!g.partition) pbuf = std::max(pbuf, (size_t)g.Np * c->Nt * g.p);
  }
  c->svw.resize(1);
  int rc;
  void* base = nullptr;
  if ((rc = dalloc(c, &base, need))) return rc;
  c->svw[0].gram = reinterpret_cast<cf*>(base);
  if (pbuf) {
    if ((rc = dalloc(c, (void**)&c->d_pbuf, pbuf * sizeof(cf)))) return rc;
    c->pbuf_elems = pbuf;
  }
  if ((rc = dalloc(c, (void**)&c->d_img_tmp, (size_t)c->Nt * c->nvox * sizeof(cf)))) return rc;
  size_t maxsm = 0;
  for (auto& g : c->scales) maxsm = std::max(maxsm, eig_smem(g.n));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_eig, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)std::max<size_t>(maxsm, 48 * 1024)));
  return MSLR_OK;
}

int patch_svst(Ctx* c, int s, const double* thr_dev, double lam, const cf* img_in, cf* img_out,
               cudaStream_t st) {
  const ScaleGeom& g = c->scales[s];
  const PatchMap m = map_of(g, c->N, c->Nt, c->nvox);
  const int nsplit = choose_split(g.Np, g.n, g.L);
  WorkPtrs w = carve(c->svw[0].gram, g.Np, g.n, nsplit);
  int rc;
  if (g.partition) {
    cf* dst = img_out;
    if (img_in == img_out) dst = c->d_img_tmp;   // Gram/rebuild read the input throughout
    if ((rc = svst_core(img_in, m, g.Np, w, nsplit, thr_dev, 0, lam, dst, 1, st, &c->launches))) return rc;
    if (dst != img_out)
      MSLR_CUDA_TRY(cudaMemcpyAsync(img_out, dst, (size_t)c->Nt * c->nvox * sizeof(cf),
                                    cudaMemcpyDeviceToDevice, st));
  } else {
    if ((rc = svst_core(img_in, m, g.Np, w, nsplit, thr_dev, 0, lam, c->d_pbuf, 0, st, &c->launches))) return rc;
    k_recombine<<<1184, 256, 0, st>>>(c->d_pbuf, m, g.d_cover, img_out);
    MSLR_CUDA_TRY(cudaGetLastError());
    c->launches += 1;
  }
  return MSLR_OK;
}

// ---------------------------------------------------------------------------
// context-free entry points
// ---------------------------------------------------------------------------
int patches_op(const int N[3], int Nt, const int ps[3], const int ss[3], const cf* src, cf* dst,
               bool to_patches, cudaStream_t st) {
  ScaleGeom g;
  int rc = geom_build(N, Nt, ps, ss, &g);
  if (rc) return rc;
  if ((rc = geom_upload(&g, N))) {
    geom_free(&g);
    return rc;
  }
  const int64_t nvox = (int64_t)N[0] * N[1] * N[2];
  const PatchMap m = map_of(g, N, Nt, nvox);
  if (to_patches) {
    const int64_t total = g.Np * Nt * (int64_t)g.p;
    k_img2patches<<<1184, 256, 0, st>>>(src, m, dst, total);
  } else {
    k_recombine<<<1184, 256, 0, st>>>(src, m, g.d_cover, dst);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  geom_free(&g);
  if (e != cudaSuccess) return fail(MSLR_ERR_CUDA, cudaGetErrorString(e));
  return MSLR_OK;
}

size_t svst_batch_bytes(int mrows, int ncols, int batch) {
  const int n = std::min(mrows, ncols);
  return eig_work_bytes(batch, n, 1) + (size_t)batch * sizeof(double) + 256 +
         (size_t)batch * mrows * ncols * sizeof(cf) + 256;
}

int svst_batch(int mrows, int ncols, int batch, const double* betas, const cf* in, cf* out,
               void* ws, size_t ws_bytes, cudaStream_t st) {
  const int n = std::min(mrows, ncols);
  const size_t need = svst_batch_bytes(mrows, ncols, batch);
  if (ws_bytes < need) return fail(MSLR_ERR_ARG, "workspace too small for mslr_svst_batch");
  WorkPtrs w = carve(ws, batch, n, 1);
  unsigned char* tail = reinterpret_cast<unsigned char*>(ws) + eig_work_bytes(batch, n, 1);
  tail = reinterpret_cast<unsigned char*>(((uintptr_t)tail + 255) & ~(uintptr_t)255);
  double* d_beta = reinterpret_cast<double*>(tail);
  tail += ((size_t)batch * sizeof(double) + 255) & ~(size_t)255;
  cf* stage = reinterpret_cast<cf*>(tail);
  MSLR_CUDA_TRY(cudaMemcpyAsync(d_beta, betas, batch * sizeof(double), cudaMemcpyHostToDevice, st));
  PatchMap m;
  m.Nx = mrows;
  m.Ny = 1;
  m.Nz = 1;
  m.nvox = mrows;
  m.Nt = ncols;
  m.psx = mrows;
  m.psy = 1;
  m.psz = 1;
  m.nx = m.ny = m.nz = 1;
  m.starts = nullptr;
  m.p = mrows;
  m.n = n;
  m.L = std::max(mrows, ncols);
  m.tall = mrows >= ncols;
  m.batch = 1;
  m.mstride = (int64_t)mrows * ncols;
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_eig, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)std::max<size_t>(eig_smem(1024), 48 * 1024)));
  const cf* src = in;
  if (in == out) {
    MSLR_CUDA_TRY(cudaMemcpyAsync(stage, in, (size_t)batch * mrows * ncols * sizeof(cf),
                                  cudaMemcpyDeviceToDevice, st));
    src = stage;
  }
  return svst_core(src, m, batch, w, 1, d_beta, 1, 1.0, out, 1, st, nullptr);
}

// ---------------------------------------------------------------------------
// Batched SVST without any allocation, for callers that cannot call
// cudaMalloc (see mslr_svst_batch_noalloc in include/mslr.h).  Its scratch is
// this file-scope device array: every GPU that loads the library holds it
// until the process exits, and all calls share it.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[MSLR_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch, looked up once per device.  In host
// code the symbol name is only a host-side stand-in, so the kernels must be
// given the address that cudaGetSymbolAddress returns for the current device.
static void* g_noalloc_addr[64];
static std::mutex g_noalloc_mu;

int svst_batch_noalloc(int mrows, int ncols, int batch, const double* betas, const cf* in, cf* out,
                       cudaStream_t st) {
  const size_t need = svst_batch_bytes(mrows, ncols, batch);
  if (need > (size_t)MSLR_NOALLOC_SCRATCH_BYTES)
    return fail(MSLR_ERR_ARG,
                "mslr_svst_batch_noalloc: this batch needs " + std::to_string(need) +
                    " bytes of scratch, more than the fixed " +
                    std::to_string((size_t)MSLR_NOALLOC_SCRATCH_BYTES) +
                    " bytes; use mslr_svst_batch with a caller workspace or split the batch");
  int dev = 0;
  MSLR_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(MSLR_ERR_UNSUPPORTED, "device ordinal above 63");
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return fail(MSLR_ERR_CUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") +
                                       cudaGetErrorString(e));
      g_noalloc_addr[dev] = p;
    }
    scratch = g_noalloc_addr[dev];
  }
  // No part of the scratch has to start at zero: every stage writes what the
  // next one reads, so the previous call's contents are simply overwritten.
  return svst_batch(mrows, ncols, batch, betas, in, out, scratch, (size_t)MSLR_NOALLOC_SCRATCH_BYTES,
                    st);
}

}  // namespace mslr
