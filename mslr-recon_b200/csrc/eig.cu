// eig.cu — per-patch Hermitian eigen stage of the patch SVST (sm_100a).
//
// For each patch Gram matrix G (n × n, Hermitian, column-major, FP32 complex)
// and threshold β this computes the scaled eigenvector matrix
//     Ṽ = V diag(√h),   h_i = max(√λ_i − β, 0) / √λ_i,
// over the eigenpairs (λ_i, v_i) of G with λ_i > β², so that the rebuild
// matrix of the patch SVST (src/recon.jl:183-211, expressed through its Gram
// matrix) is W = Ṽ Ṽᴴ — one more Gram product, formed by the batched Gram
// kernels after this launch.  One CTA per patch — 384 threads when n <= 384
// (two patches per SM, so one patch's latency-bound phases overlap the
// other's), else 1024; one launch may cover several segments (the patches of
// several scales, each with its own n and λ_k).  The matrix lives in global
// memory (L2); only its lower triangle is read or written:
//   1. Householder tridiagonalisation G = Q T Qᴴ (FP32).  Each step applies
//      the previous step's rank-2 update on the fly while forming the next
//      Hermitian matrix-vector product over 32 × 32 tiles of the trailing
//      lower triangle (one warp per tile: row sums per lane, column sums by a
//      shuffle transpose-reduction, both stored per tile and summed per row
//      in a fixed order, so results are bit-reproducible), streaming the
//      trailing triangle once per step; the working set of ~300 resident
//      patches stays in L2.  The pass also leaves the next column in shared
//      memory, and every thread computes the reflector scalars and the next
//      pivot row's (v, w) itself, so a step has four block barriers.
//   2. Eigenvalues of T above β² by bisection on FP64 Sturm counts, one
//      thread per eigenvalue.
//   3. Eigenvectors of T by FP64 twisted factorisation, one thread per
//      eigenvector; eigenvalues equal to working precision (true
//      degeneracies) are re-orthogonalised cooperatively by Gram–Schmidt.
//   4. V = Q Z with the reflectors applied 16 at a time in compact WY form
//      (Q_b = I − Y T Yᴴ); thread i keeps vector i's block coefficients in
//      registers, so the update needs no cross-thread reduction.
//   5. Ṽ written as conj(V) diag(√h) in row-major order ([row][vector]),
//      columns beyond the rank set to zero.
// Zero patches give no eigenvalue above β² and Ṽ = 0, hence W = 0 (the
// reference's zero-norm skip, src/recon.jl:185).
//
// Split stage (thresholded SVSTs with 64 <= n <= 384): three launches instead
// of one, so that each phase runs at the occupancy it needs — phase 1 and the
// WY blocks' T factors (two CTAs per SM), phases 2–3 (four CTAs per SM, all
// patches resident at once), and phases 4–5 as k_wy_apply: 32 eigenvectors
// of one patch per CTA, held in registers through every block update.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "internal.h"

namespace mslr {

namespace {

constexpr int kT = 1024;   // most threads per CTA (one row / eigenvalue per thread)
constexpr int kSmallT = 384;   // CTA size for n <= 384: two patches share an SM
constexpr int kNb = 16;    // reflectors per WY block
constexpr int kCW = 16;    // eigenvectors per back-transform pass
constexpr int kPairsMinB = 4;   // CTAs per SM of the split stage's eigenpair launch

__device__ __forceinline__ float warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block sums; every thread gets the result.  Consecutive calls must alternate
// between two scratch buffers (one barrier per call).
__device__ __forceinline__ float block_sum(float v, float* red) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float r = 0.f;
  const int nw = (int)(blockDim.x >> 5);
  for (int i = 0; i < nw; ++i) r += red[i];
  return r;
}
__device__ __forceinline__ double block_sum_d(double v, double* red) {
  v = warp_sum_d(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  const int nw = (int)(blockDim.x >> 5);
  for (int i = 0; i < nw; ++i) r += red[i];
  return r;
}

// eigenvalues of the symmetric tridiagonal (d, e²) strictly below x
__device__ __forceinline__ int sturm_less(const double* d, const double* e2, int n, double x,
                                          double pivmin) {
  int cnt = 0;
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += (q < 0.0);
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += (q < 0.0);
  }
  return cnt;
}

// sturm_less in FP32 on a copy of T scaled to norm ~1 (d / ‖T‖, e² / ‖T‖²),
// with the fast reciprocal division: the count is exact for a matrix within a
// few FP32 roundings of T (the Sturm sequence is backward stable), which is
// all the first rounds of bracketing need
__device__ __forceinline__ int sturm_less_f(const float* d, const float* e2, int n, float x) {
  constexpr float pivmin = 1e-30f;
  int cnt = 0;
  float q = d[0] - x;
  if (fabsf(q) < pivmin) q = -pivmin;
  cnt += (q < 0.f);
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - __fdividef(e2[i - 1], q);
    if (fabsf(q) < pivmin) q = -pivmin;
    cnt += (q < 0.f);
  }
  return cnt;
}

struct Seg {
  int n;
  int64_t first;   // first block of the segment
  int64_t np;      // patches
  cf* gram;        // np × n × n: G in (lower triangle), Householder vectors out
  cf* zv;          // np × n × n: eigenvectors, [row j][vector i], i fastest; Ṽ out
  double* aux;     // np × n × n: FP64 pivots of the twisted factorisations
  int* rank;       // np
  double lam;      // threshold multiplier of the segment (λ_k)
  double* nuc;     // values-only mode when set: np sums Σ √λ_i over λ_i above β², no vectors
  double* lam_out; // full mode when set: all n eigenpairs, V unscaled in zv, λ (descending) here
  double* side;    // split stage: np × 6n — d, e (FP64), λ, h of the tridiagonal (k_eig modes 1, 2)
};

constexpr int kMaxSeg = 8;

struct EigArgs {
  int nseg;
  Seg seg[kMaxSeg];
  const double* thr;   // device: threshold scale (ζ or β), or per patch
  int thr_per_patch;
  int rz;              // eigenvectors staged in shared memory (more: global slots)
};

// vectors are padded to n + 32 entries (zero tails) so 32-wide tiles read them in bounds
// Per-tile partial sums of the tridiagonalisation's matvec: 64 values for
// each 32 × 32 tile of the largest trailing triangle (side n − 1).
size_t part_bytes(int n) {
  const size_t T = (size_t)(n - 1 + 31) / 32;
  return T * (T + 1) / 2 * 64 * sizeof(cf);
}

size_t vec_bytes(int n) {
  const size_t np = (size_t)n + 32;
  return np * sizeof(float4) + 5 * np * sizeof(cf) + 4 * (size_t)n * sizeof(double) +
         3 * (size_t)n * sizeof(float) + 64 * sizeof(float) + 64 * sizeof(double);
}

// Buffers of the back-transform besides the vector stage: Y (n × kNb), T and
// YᴴY (kNb × kNb each), S and T·S (kNb × kCW each), one partial sum per thread.
size_t wy_bytes(int n, int threads) {
  return ((size_t)n * kNb + 2 * kNb * kNb + 2 * kNb * kCW + (size_t)threads + 1) * sizeof(cf);
}

// The region after the vectors, by phase: the matvec partial sums (phase 1,
// 384-thread variant), the FP64 twisted-factorisation columns of up to rz
// eigenvectors (phase 3: z and D+, n × rz doubles each), the complex
// eigenvector stage (n × rz) followed by the back-transform buffers (phase 4).
size_t smem_bytes(int n, int threads, int rz) {
  const size_t stage = (size_t)n * rz * sizeof(cf);
  size_t region = std::max(2 * stage, stage + wy_bytes(n, threads));
  if (threads <= kSmallT) region = std::max(region, part_bytes(n));
  return vec_bytes(n) + region + 128;
}

// Dynamic shared memory one CTA may use: two CTAs per SM for the 384-thread
// variant (228 KB per SM, 1 KB reserved per CTA), one for the large variant;
// both leave room for the kernel's static shared variables.
size_t smem_budget(int threads) { return threads <= kSmallT ? 112 * 1024 : 227 * 1024 - 1024; }

// eigenvectors staged in shared memory: the most that fit beside everything else
int stage_cols(int n, int threads) {
  int rz = 0;
  while (rz < n && smem_bytes(n, threads, rz + 1) <= smem_budget(threads)) ++rz;
  return rz;
}

__device__ __forceinline__ unsigned long long pk2(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long u) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(u));
  return v;
}
// (a.x·b.x + c.x, a.y·b.y + c.y), each lane one correctly rounded FMA
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b,
                                                   unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// Eight columns of a tile row: the pending rank-2 update of element
// (row, jb + b), its contribution to the row sum y_row and to the column
// partials (cr, ci), written back.
__device__ __forceinline__ void tile_group(cf* a, const float4* pw, const float4* vv, cf vpr, cf wpr, cf vr,
                                           float& yr, float& yim, float* cr, float* ci) {
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const float4 p = pw[b];   // (vp_j, wp_j)
    const float4 v2 = vv[b >> 1];
    const float vjx = (b & 1) ? v2.z : v2.x, vjy = (b & 1) ? v2.w : v2.y;
    cf e = a[b];
    e.x -= (vpr.x * p.z + vpr.y * p.w) + (wpr.x * p.x + wpr.y * p.y);
    e.y -= (vpr.y * p.z - vpr.x * p.w) + (wpr.y * p.x - wpr.x * p.y);
    a[b] = e;
    yr += e.x * vjx - e.y * vjy;
    yim += e.x * vjy + e.y * vjx;
    cr[b] = e.x * vr.x + e.y * vr.y;
    ci[b] = e.x * vr.y - e.y * vr.x;
  }
}

// Column sums of eight columns over the 32 lanes (a shuffle transpose): lane l
// ends with the sum of column l / 4 in cr[0], ci[0].
__device__ __forceinline__ void col_sums(float* cr, float* ci, int lane) {
  const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float sr_ = h16 ? cr[q] : cr[q + 4], si_ = h16 ? ci[q] : ci[q + 4];
    const float kr = h16 ? cr[q + 4] : cr[q], ki = h16 ? ci[q + 4] : ci[q];
    cr[q] = kr + __shfl_xor_sync(0xffffffffu, sr_, 16);
    ci[q] = ki + __shfl_xor_sync(0xffffffffu, si_, 16);
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const float sr_ = h8 ? cr[q] : cr[q + 2], si_ = h8 ? ci[q] : ci[q + 2];
    const float kr = h8 ? cr[q + 2] : cr[q], ki = h8 ? ci[q + 2] : ci[q];
    cr[q] = kr + __shfl_xor_sync(0xffffffffu, sr_, 8);
    ci[q] = ki + __shfl_xor_sync(0xffffffffu, si_, 8);
  }
  {
    const float sr_ = h4 ? cr[0] : cr[1], si_ = h4 ? ci[0] : ci[1];
    const float kr = h4 ? cr[1] : cr[0], ki = h4 ? ci[1] : ci[0];
    cr[0] = kr + __shfl_xor_sync(0xffffffffu, sr_, 4);
    ci[0] = ki + __shfl_xor_sync(0xffffffffu, si_, 4);
  }
  cr[0] += __shfl_xor_sync(0xffffffffu, cr[0], 2);
  ci[0] += __shfl_xor_sync(0xffffffffu, ci[0], 2);
  cr[0] += __shfl_xor_sync(0xffffffffu, cr[0], 1);
  ci[0] += __shfl_xor_sync(0xffffffffu, ci[0], 1);
}

// An off-diagonal tile (I, J), J < I, whose 32 columns all lie inside the
// matrix (rows past n, in the last tile row, are masked per lane): the same
// arithmetic as the general tile path without its per-element tests; the
// column values come from the re-based vectors as
// 16-byte loads, and each group's loads are issued before the previous
// group is updated and stored (they address other columns) when PIPE (the
// 384-thread variant; the 1024-thread variant's 64 registers do not hold
// the second group).
template <bool PIPE>
__device__ __noinline__ void full_tile(cf* A, int n, int o, int I, int J, int t, int lane, const float4* spw,
                                       const cf* svr, const cf* svp, const cf* swp, const cf* sv, cf* part,
                                       cf* scol) {
  const int row = o + I * 32 + lane;
  const bool rowok = row < n;   // the last tile row may reach past n (its vectors are zero there)
  const cf vpr = svp[row], wpr = swp[row], vr = sv[row];
  float yr = 0.f, yim = 0.f;
  const int jo = J * 32;   // first column − o
  cf* col0 = A + (int64_t)(o + jo) * n + row;
  const float4* pw = spw + jo;
  const float4* vv = reinterpret_cast<const float4*>(svr + jo);
  cf a[8];
  if constexpr (PIPE) {
#pragma unroll
    for (int b = 0; b < 8; ++b) a[b] = rowok ? __ldcg(col0 + (int64_t)b * n) : make_float2(0.f, 0.f);
  }
#pragma unroll 1
  for (int g8 = 0; g8 < 4; ++g8) {
    cf nx[8];
    if constexpr (PIPE) {
      if (g8 < 3) {
#pragma unroll
        for (int b = 0; b < 8; ++b)
          nx[b] = rowok ? __ldcg(col0 + (int64_t)((g8 + 1) * 8 + b) * n) : make_float2(0.f, 0.f);
      }
    } else {
#pragma unroll
      for (int b = 0; b < 8; ++b) a[b] = rowok ? __ldcg(col0 + (int64_t)(g8 * 8 + b) * n) : make_float2(0.f, 0.f);
    }
    float cr[8], ci[8];
    tile_group(a, pw + g8 * 8, vv + g8 * 4, vpr, wpr, vr, yr, yim, cr, ci);
    if (scol && g8 == 0) scol[row] = a[0];   // column o, the next step's
    if (rowok) {
#pragma unroll
      for (int b = 0; b < 8; ++b) col0[(int64_t)(g8 * 8 + b) * n] = a[b];
    }
    col_sums(cr, ci, lane);
    if ((lane & 3) == 0) part[(2 * t + 1) * 32 + g8 * 8 + (lane >> 2)] = make_float2(cr[0], ci[0]);
    if constexpr (PIPE) {
#pragma unroll
      for (int b = 0; b < 8; ++b) a[b] = nx[b];
    }
  }
  part[2 * t * 32 + lane] = make_float2(yr, yim);
}

// One eigenvector in global memory (column `col` of Z, row stride n) through
// one WY block of kNb reflectors starting at row k0 + 1: S = Yᴴ z, S ← T S,
// z −= Y S.  Y's rows are read as 16-byte pairs (sYb is 16-byte aligned) and
// the vector's elements kB rows ahead of their use.
__device__ __noinline__ void bt_vector(cf* Z, int n, int col, int k0, const cf* sYb, const cf* sT) {
  cf Sv[kNb];
#pragma unroll
  for (int jj = 0; jj < kNb; ++jj) Sv[jj] = make_float2(0.f, 0.f);
  constexpr int kB = 4;
  auto accum = [&](int row, const cf z) {
    const float4* y4 = reinterpret_cast<const float4*>(sYb + row * kNb);
#pragma unroll
    for (int q = 0; q < kNb / 2; ++q) {
      const float4 yy = y4[q];
      Sv[2 * q].x += yy.x * z.x + yy.y * z.y;
      Sv[2 * q].y += yy.x * z.y - yy.y * z.x;
      Sv[2 * q + 1].x += yy.z * z.x + yy.w * z.y;
      Sv[2 * q + 1].y += yy.z * z.y - yy.w * z.x;
    }
  };
  {
    int row = k0 + 1;
    for (; row + kB <= n; row += kB) {
      cf z[kB];
#pragma unroll
      for (int b = 0; b < kB; ++b) z[b] = __ldcg(Z + (int64_t)(row + b) * n + col);
#pragma unroll
      for (int b = 0; b < kB; ++b) accum(row + b, z[b]);
    }
    for (; row < n; ++row) accum(row, __ldcg(Z + (int64_t)row * n + col));
  }
  // T upper-triangular: S[a] is last needed by row a itself (in place)
#pragma unroll
  for (int a = 0; a < kNb; ++a) {
    cf sacc = make_float2(0.f, 0.f);
#pragma unroll
    for (int b = a; b < kNb; ++b) sacc = cadd(sacc, cmul(sT[a * kNb + b], Sv[b]));
    Sv[a] = sacc;
  }
  auto upd = [&](int row, cf z) {
    const float4* y4 = reinterpret_cast<const float4*>(sYb + row * kNb);
#pragma unroll
    for (int q = 0; q < kNb / 2; ++q) {
      const float4 yy = y4[q];
      z = csub(z, cmul(make_float2(yy.x, yy.y), Sv[2 * q]));
      z = csub(z, cmul(make_float2(yy.z, yy.w), Sv[2 * q + 1]));
    }
    return z;
  };
  int row = k0 + 1;
  for (; row + kB <= n; row += kB) {
    cf z[kB];
#pragma unroll
    for (int b = 0; b < kB; ++b) z[b] = __ldcg(Z + (int64_t)(row + b) * n + col);
#pragma unroll
    for (int b = 0; b < kB; ++b) z[b] = upd(row + b, z[b]);
#pragma unroll
    for (int b = 0; b < kB; ++b) Z[(int64_t)(row + b) * n + col] = z[b];
  }
  for (; row < n; ++row) Z[(int64_t)row * n + col] = upd(row, Z[(int64_t)row * n + col]);
}

// Upper-triangle slot q (column by column, column c holding rows 0..c−1) of a
// column-major n × n matrix: the split stage keeps the WY blocks' T factors in
// the strictly upper triangle of the patch's Gram buffer, which nothing reads
// between the tridiagonalisation and the back-transform (the W Gram rewrites
// the whole buffer afterwards).
__device__ __forceinline__ int64_t upper_slot(int n, int q) {
  int c = (int)((1.f + sqrtf(1.f + 8.f * (float)q)) * 0.5f);
  while (c > 1 && c * (c - 1) / 2 > q) --c;
  while ((c + 1) * c / 2 <= q) ++c;
  return (int64_t)c * n + (q - c * (c - 1) / 2);
}

// T factors (zlarft, forward columnwise) of the WY blocks of kNb reflectors,
// taken from the last reflector down as the back-transform applies them;
// block blk = (n − 1 − kend) / kNb goes to upper slots [256·blk, 256·blk + 256).
// sYb: n × kNb complex scratch followed by two kNb × kNb blocks.
__device__ void wy_factors(cf* A, int n, const float* taur, const float* taui, cf* sYb, int tid, int kT) {
  cf* sT = sYb + (int64_t)n * kNb;
  cf* sYY = sT + kNb * kNb;
  const int nref = n - 1;
  for (int kend = nref; kend > 0; kend -= kNb) {
    const int k0 = max(0, kend - kNb);
    const int nb = kend - k0;
    const int blk = (nref - kend) / kNb;
    const int m = n - k0 - 1;
    for (int q = tid; q < m * kNb; q += kT) {   // rows k0+1 .. n−1 of reflectors k0 .. k0+nb−1
      const int jj = q / m, row = k0 + 1 + (q - jj * m);
      const int k = k0 + jj;
      cf y = make_float2(0.f, 0.f);
      if (jj < nb) {
        if (row == k + 1) y = make_float2(1.f, 0.f);
        else if (row > k + 1) y = __ldcg(A + (int64_t)k * n + row);
      }
      sYb[row * kNb + jj] = y;
    }
    __syncthreads();
    if (tid < kNb * kNb) {   // Yᴴ Y
      const int a = tid / kNb, b = tid - a * kNb;
      float sr = 0.f, si = 0.f;
      for (int row = k0 + 1; row < n; ++row) {
        const cf ya = sYb[row * kNb + a], yb = sYb[row * kNb + b];
        sr += ya.x * yb.x + ya.y * yb.y;
        si += ya.x * yb.y - ya.y * yb.x;
      }
      sYY[tid] = make_float2(sr, si);
    }
    __syncthreads();
    if (tid < 32) {   // lane a owns row a of T
      const int a = tid;
      for (int jj = 0; jj < kNb; ++jj) {
        const cf tj = (jj < nb) ? make_float2(taur[k0 + jj], taui[k0 + jj]) : make_float2(0.f, 0.f);
        if (a < jj) {
          cf sacc = make_float2(0.f, 0.f);
          for (int b = a; b < jj; ++b) sacc = cadd(sacc, cmul(sT[a * kNb + b], sYY[b * kNb + jj]));
          const cf v = cmul(tj, sacc);
          sT[a * kNb + jj] = make_float2(-v.x, -v.y);
        } else if (a < kNb) {
          sT[a * kNb + jj] = (a == jj) ? tj : make_float2(0.f, 0.f);
        }
        __syncwarp();
      }
    }
    __syncthreads();
    for (int t = tid; t < kNb * kNb; t += kT) A[upper_slot(n, blk * kNb * kNb + t)] = sT[t];
    __syncthreads();
  }
}

// MODE 0: the whole stage in one launch.  The split stage (three launches):
// MODE 1 tridiagonalises and writes d, e to the side buffer and the WY
// blocks' T factors to the Gram's upper triangle; MODE 2 computes the
// eigenpairs of T from the side buffer (vectors into zv, FP32, [row][vector],
// λ and h back to the side buffer); k_wy_apply then forms Ṽ.
template <int MAXT, int MINB, int MODE>
__global__ void __launch_bounds__(MAXT, MINB) k_eig(EigArgs g) {
  extern __shared__ __align__(16) unsigned char smraw[];
  int s = 0;
  while (s + 1 < g.nseg && (int64_t)blockIdx.x >= g.seg[s + 1].first) ++s;
  const Seg& S = g.seg[s];
  const int n = S.n;
  const int64_t ip = (int64_t)blockIdx.x - S.first;
  const int tid = threadIdx.x;
  const int kT = blockDim.x;   // n <= blockDim.x
  cf* A = S.gram + ip * (int64_t)n * n;
  cf* Z = S.zv + ip * (int64_t)n * n;
  double* AUX = S.aux + ip * (int64_t)n * n;

  // shared layout (8-byte aligned pieces first); complex vectors hold n + 32 entries
  const int npad = n + 32;
  double* dd = reinterpret_cast<double*>(smraw);   // diagonal        [n]
  double* ee = dd + n;                              // off-diagonal    [n]
  double* ee2 = ee + n;                             // e²              [n]
  double* lam = ee2 + n;                            // eigenvalues     [n]
  double* redd = lam + n;                           // 64 doubles
  // the step's vectors again, indexed from the trailing block's first row o =
  // k + 1 (16-byte aligned, so a tile's eight columns load as vectors):
  // spw[j − o] = (vp_j, wp_j), svr[j − o] = v_j
  float4* spw = reinterpret_cast<float4*>(redd + 64);   //             [npad]
  cf* svr = reinterpret_cast<cf*>(spw + npad);           //             [npad]
  cf* sv = svr + npad;                              // v of this step  [npad]
  cf* svp = sv + npad;                              // previous v      [npad]
  cf* swp = svp + npad;                             // previous w      [npad]
  cf* scol = swp + npad;                            // next column     [npad]
  float* hv = reinterpret_cast<float*>(scol + npad); // h              [n]
  float* taur = hv + n;                             // τ               [n]
  float* taui = taur + n;                           //                 [n]
  float* red0 = taui + n;                           // 2 × 32 floats
  float* red1 = red0 + 32;
  cf* sY = reinterpret_cast<cf*>((reinterpret_cast<uintptr_t>(red1 + 32) + 15) & ~(uintptr_t)15);
  __shared__ cf s_x;
  __shared__ double s_bd[4];
  __shared__ int s_r;

  const bool full = S.lam_out != nullptr;
  const double beta_d = full ? 0.0 : g.thr[g.thr_per_patch ? (int64_t)blockIdx.x : 0] * S.lam;
  const float beta = (float)beta_d;
  (void)beta;

  const int i = tid;   // row owned by this thread (n <= kT)
  const int warp = tid >> 5, lane = tid & 31, nwarp = kT >> 5;
  if constexpr (MODE == 2) {   // T from the side buffer (the same FP64 values phase 1 keeps)
    const double* side = S.side + ip * 6 * (int64_t)n;
    for (int q = tid; q < n; q += kT) {
      dd[q] = side[q];
      const double e = side[n + q];
      ee[q] = e;
      ee2[q] = e * e;
    }
    (void)nwarp;
    __syncthreads();
  } else {
  // ---- 1. tridiagonalisation with delayed rank-2 updates ---------------------
  for (int q = tid; q < npad; q += kT) {
    sv[q] = make_float2(0.f, 0.f);
    svp[q] = make_float2(0.f, 0.f);
    swp[q] = make_float2(0.f, 0.f);
    svr[q] = make_float2(0.f, 0.f);
    spw[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  // per-tile row / column sums of the Hermitian matvec of a step: shared
  // memory (sharing the WY blocks' storage) for the 384-thread variant, the
  // patch's FP64 pivot scratch (idle until phase 3) for the large variant
  cf* part = (MAXT <= kSmallT) ? sY : reinterpret_cast<cf*>(AUX);
  // (vp, wp) of the pivot row k, known to every thread: row k's entries of the
  // previous step's v (1 when it reflected) and w (τ y_k − c), the latter from
  // the row sums every thread adds up itself, so no barrier publishes them
  cf vpk = make_float2(0.f, 0.f), wpk = make_float2(0.f, 0.f);
  for (int k = 0; k < n - 1; ++k) {
    // current column k and diagonal k: stored − (vp wpᴴ + wp vpᴴ); after the
    // first step the previous pass left the stored column in scol
    cf x = make_float2(0.f, 0.f);
    cf vpi = make_float2(0.f, 0.f), wpi = make_float2(0.f, 0.f);
    if (i < n) {
      vpi = svp[i];
      wpi = swp[i];
    }
    if (i >= k && i < n) {
      x = (k == 0) ? __ldcg(A + i) : scol[i];
      x = csub(x, cadd(cmul(vpi, cconj(wpk)), cmul(wpi, cconj(vpk))));
      if (i == k) dd[k] = (double)x.x;
    }
    if (i == k + 1) s_x = x;
    const float xn = block_sum((i >= k + 2 && i < n) ? cabs2(x) : 0.f, red0);
    // zlarfg, by every thread on the same values: Hᴴ (α, x) = (β, 0), H = I − τ v vᴴ, β real
    float tr, ti, sr, si;
    {
      const float ar = s_x.x, ai = s_x.y;
      float bt;
      if (xn == 0.f && ai == 0.f) {
        bt = ar;
        tr = ti = 0.f;
        sr = 1.f;
        si = 0.f;
      } else {
        bt = -copysignf(sqrtf(ar * ar + ai * ai + xn), ar);
        tr = (bt - ar) / bt;
        ti = -ai / bt;
        const float zr = ar - bt, zi = ai;
        const float den = zr * zr + zi * zi;
        sr = zr / den;
        si = -zi / den;
      }
      if (i == k + 1) {
        ee[k] = (double)bt;
        ee2[k] = (double)bt * (double)bt;
        taur[k] = tr;
        taui[k] = ti;
      }
    }
    const cf tau = make_float2(tr, ti);
    const cf scal = make_float2(sr, si);
    const bool refl = (tau.x != 0.f || tau.y != 0.f);
    cf vi = make_float2(0.f, 0.f);
    if (i == k + 1) {
      vi = make_float2(1.f, 0.f);
    } else if (i >= k + 2 && i < n) {
      vi = cmul(x, scal);
      A[(int64_t)k * n + i] = vi;   // reflector kept below the subdiagonal
    }
    if (i < n) sv[i] = vi;
    if (i > k && i < n) svr[i - k - 1] = vi;
    __syncthreads();
    // fused over the trailing lower triangle [o, n)²: A22 ← A22 − (vp wpᴴ + wp vpᴴ)
    // and y = A22 v (Hermitian: element (r, c), r > c, also gives y_c += conj(a) v_r).
    {
      const int o = k + 1;
      const int T = (n - o + 31) >> 5;
      const int ntile = T * (T + 1) / 2;
      // work order: the T diagonal tiles (the costlier general path) first,
      // one per warp, then the off-diagonal tiles row by row; t is the
      // tile's slot in the partial sums (row-major over the triangle)
      for (int u = warp; u < ntile; u += nwarp) {
        int I, J;
        if (u < T) {
          I = J = u;
        } else {
          const int q = u - T;   // q-th tile strictly below the diagonal
          I = (int)((1.f + sqrtf(8.f * (float)q + 1.f)) * 0.5f);
          while (I > 1 && I * (I - 1) / 2 > q) --I;
          while ((I + 1) * I / 2 <= q) ++I;
          J = q - I * (I - 1) / 2;
        }
        const int t = I * (I + 1) / 2 + J;
        if (I != J) {   // off-diagonal tiles: every column inside the matrix
          full_tile<(MAXT <= kSmallT)>(A, n, o, I, J, t, lane, spw, svr, svp, swp, sv, part,
                                       J == 0 ? scol : nullptr);
          continue;
        }
        const bool diag = (I == J);
        const int row = o + I * 32 + lane;
        const bool rowok = row < n;
        const int rr = rowok ? row : n - 1;
        const cf vpr = svp[rr], wpr = swp[rr];
        const cf vr = rowok ? sv[rr] : make_float2(0.f, 0.f);
        float yr = 0.f, yim = 0.f;
        const int j0 = o + J * 32;
        cf* col0 = A + (int64_t)j0 * n + rr;
        for (int g8 = 0; g8 < 4; ++g8) {
          const int jb = j0 + g8 * 8;
          if (jb >= n) break;
          cf a[8];
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            const int j = jb + b;
            const bool ok = rowok && j < n && (!diag || row >= j);
            a[b] = ok ? __ldcg(col0 + (int64_t)(g8 * 8 + b) * n) : make_float2(0.f, 0.f);
          }
          float cr[8], ci[8];
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            const int j = jb + b;
            const bool ok = rowok && j < n && (!diag || row >= j);
            const cf vpj = svp[j], wpj = swp[j], vj = sv[j];
            cf e = a[b];
            e.x -= (vpr.x * wpj.x + vpr.y * wpj.y) + (wpr.x * vpj.x + wpr.y * vpj.y);
            e.y -= (vpr.y * wpj.x - vpr.x * wpj.y) + (wpr.y * vpj.x - wpr.x * vpj.y);
            if (!ok) e = make_float2(0.f, 0.f);
            a[b] = e;
            yr += e.x * vj.x - e.y * vj.y;
            yim += e.x * vj.y + e.y * vj.x;
            const bool low = !diag || row > j;   // strictly below the diagonal
            cr[b] = low ? (e.x * vr.x + e.y * vr.y) : 0.f;
            ci[b] = low ? (e.x * vr.y - e.y * vr.x) : 0.f;
          }
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            const int j = jb + b;
            if (rowok && j < n && (!diag || row >= j)) col0[(int64_t)(g8 * 8 + b) * n] = a[b];
          }
          if (J == 0 && g8 == 0 && rowok) scol[row] = a[0];   // column o, the next step's
          // column sums over the 32 lanes: lane l ends with the sum of column l/4
          const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const float sr_ = h16 ? cr[q] : cr[q + 4], si_ = h16 ? ci[q] : ci[q + 4];
            const float kr = h16 ? cr[q + 4] : cr[q], ki = h16 ? ci[q + 4] : ci[q];
            cr[q] = kr + __shfl_xor_sync(0xffffffffu, sr_, 16);
            ci[q] = ki + __shfl_xor_sync(0xffffffffu, si_, 16);
          }
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const float sr_ = h8 ? cr[q] : cr[q + 2], si_ = h8 ? ci[q] : ci[q + 2];
            const float kr = h8 ? cr[q + 2] : cr[q], ki = h8 ? ci[q + 2] : ci[q];
            cr[q] = kr + __shfl_xor_sync(0xffffffffu, sr_, 8);
            ci[q] = ki + __shfl_xor_sync(0xffffffffu, si_, 8);
          }
          {
            const float sr_ = h4 ? cr[0] : cr[1], si_ = h4 ? ci[0] : ci[1];
            const float kr = h4 ? cr[1] : cr[0], ki = h4 ? ci[1] : ci[0];
            cr[0] = kr + __shfl_xor_sync(0xffffffffu, sr_, 4);
            ci[0] = ki + __shfl_xor_sync(0xffffffffu, si_, 4);
          }
          cr[0] += __shfl_xor_sync(0xffffffffu, cr[0], 2);
          ci[0] += __shfl_xor_sync(0xffffffffu, ci[0], 2);
          cr[0] += __shfl_xor_sync(0xffffffffu, cr[0], 1);
          ci[0] += __shfl_xor_sync(0xffffffffu, ci[0], 1);
          if ((lane & 3) == 0 && jb + (lane >> 2) < n)
            part[(2 * t + 1) * 32 + g8 * 8 + (lane >> 2)] = make_float2(cr[0], ci[0]);
        }
        part[2 * t * 32 + lane] = make_float2(yr, yim);
      }
    }
    __syncthreads();
    // y_i in a fixed order: the row sums of tiles (I, 0..I), then the column
    // sums of tiles (I..T-1, I) — the same bits on every run; every thread
    // also adds up y of row k + 1 (the next pivot row) in the same order
    float yr = 0.f, yi = 0.f, y1r = 0.f, y1i = 0.f;
    {
      const int o = k + 1, T = (n - o + 31) >> 5;
      if (i >= k + 1 && i < n) {
        const int I = (i - o) >> 5, l = (i - o) & 31;
        const int t0 = I * (I + 1) / 2;
        for (int J = 0; J <= I; ++J) {
          const cf v = part[2 * (t0 + J) * 32 + l];
          yr += v.x;
          yi += v.y;
        }
        for (int I2 = I; I2 < T; ++I2) {
          const cf v = part[(2 * (I2 * (I2 + 1) / 2 + I) + 1) * 32 + l];
          yr += v.x;
          yi += v.y;
        }
      }
      {
        const cf v = part[0];
        y1r += v.x;
        y1i += v.y;
      }
      for (int I2 = 0; I2 < T; ++I2) {
        const cf v = part[(2 * (I2 * (I2 + 1) / 2)) * 32 + 32];
        y1r += v.x;
        y1i += v.y;
      }
    }
    // vᴴ y (real for Hermitian A)
    const float vy = block_sum((i >= k + 1 && i < n) ? (vi.x * yr + vi.y * yi) : 0.f, red1);
    const float c = 0.5f * (tau.x * tau.x + tau.y * tau.y) * vy;
    // the next pivot row's (vp, wp); thread k + 1 stores these same values
    if (refl) {
      const cf ty = cmul(tau, make_float2(y1r, y1i));
      vpk = make_float2(1.f, 0.f);
      wpk = make_float2(ty.x - c, ty.y);
    } else {
      vpk = wpk = make_float2(0.f, 0.f);
    }
    if (i < n) {
      cf w = make_float2(0.f, 0.f);
      if (i == k + 1) {
        w = wpk;
      } else if (i > k + 1 && refl) {
        const cf ty = cmul(tau, make_float2(yr, yi));
        w = make_float2(ty.x - c * vi.x, ty.y - c * vi.y);
      }
      swp[i] = w;
      svp[i] = refl ? vi : make_float2(0.f, 0.f);
      if (i > k + 1) {
        const cf vq = refl ? vi : make_float2(0.f, 0.f);
        spw[i - k - 2] = make_float4(vq.x, vq.y, w.x, w.y);
      }
    }
    // no barrier here: the next step reads only this thread's own svp/swp
    // entries before its first block sum, and the reduction buffers of the
    // two sums differ
  }
  if (i == n - 1) {
    cf x = __ldcg(A + (int64_t)(n - 1) * n + (n - 1));
    const cf vpk = svp[n - 1], wpk = swp[n - 1];
    x = csub(x, cadd(cmul(vpk, cconj(wpk)), cmul(wpk, cconj(vpk))));
    dd[n - 1] = (double)x.x;
    ee[n - 1] = 0.0;
    ee2[n - 1] = 0.0;
  }
  __syncthreads();
  if constexpr (MODE == 1) {
    double* side = S.side + ip * 6 * (int64_t)n;
    for (int q = tid; q < n; q += kT) {
      side[q] = dd[q];
      side[n + q] = ee[q];
    }
    wy_factors(A, n, taur, taui, sY, tid, kT);
    return;
  }
  }   // phase 1 (MODE != 2)

  // ---- 2. eigenvalues above β² (FP64 multisection) ----------------------------
  if (tid == 0) {
    double gl = dd[0], gu = dd[0], emax2 = 0.0;
    for (int q = 0; q < n; ++q) {
      const double rr = (q > 0 ? fabs(ee[q - 1]) : 0.0) + (q < n - 1 ? fabs(ee[q]) : 0.0);
      gl = fmin(gl, dd[q] - rr);
      gu = fmax(gu, dd[q] + rr);
      if (q < n - 1) emax2 = fmax(emax2, ee2[q]);
    }
    const double tnorm = fmax(fabs(gl), fabs(gu));
    const double pivmin = fmax(2.2250738585072014e-308 * fmax(emax2, 1.0), 1e-290);
    const double pad = 2.0 * 2.220446049250313e-16 * tnorm * n + pivmin;
    gl -= pad;
    gu += pad;
    s_bd[0] = gl;
    s_bd[1] = gu;
    s_bd[2] = pivmin;
    s_bd[3] = tnorm;
    const double thr2 = beta_d * beta_d;
    s_r = full ? n : (thr2 >= gu) ? 0 : n - sturm_less(dd, ee2, n, thr2, pivmin);
  }
  __syncthreads();
  const int r = s_r;
  const double gl = full ? s_bd[0] : fmax(s_bd[0], beta_d * beta_d), gu = s_bd[1],
               pivmin = s_bd[2], tnorm = s_bd[3];
  if (tid == 0) S.rank[ip] = r;
  // FP32 copy of T scaled by 1/‖T‖ (in the phase-1 vector buffers, free now)
  const double tsc = fmax(tnorm, 1e-300);
  float* ddf = reinterpret_cast<float*>(sv);
  float* e2f = ddf + n;
  for (int q = tid; q < n; q += kT) {
    ddf[q] = (float)(dd[q] / tsc);
    e2f[q] = (float)(ee2[q] / tsc / tsc);
  }
  __syncthreads();
  {
    // A group of gsz threads (a power of two, at most a warp) per eigenvalue:
    // each round counts the eigenvalues below gsz evenly spaced interior
    // points of the bracket and keeps the sub-interval holding the
    // eigenvalue, a factor gsz + 1 per round of Sturm sequences instead of
    // bisection's 2.  The first rounds run on the FP32 copy; the bracket is
    // then widened by 4e-6·‖T‖ (far beyond the FP32 counts' error), checked
    // with two FP64 counts (the whole interval again if the check fails) and
    // narrowed in FP64 to 4e-13·‖T‖ — enough for the twisted factorisations'
    // vectors, whose error scales with |λ̂ − λ| / gap.
    int gsz = 1;
    while (gsz < 32 && 2 * gsz * r <= kT) gsz <<= 1;
    const int e = tid / gsz, sl = tid & (gsz - 1);
    if (warp * 32 < r * gsz) {   // whole warps, for the shuffles
      const int kth = n - 1 - e;   // e-th largest = kth smallest
      const double frac = (double)(sl + 1) / (double)(gsz + 1);
      double lo = gl, hi = gu;
      bool done = e >= r;
      if (tnorm > 0.0) {
        const float fracf = (float)frac;
        float lof = (float)(gl / tsc), hif = (float)(gu / tsc);
        bool fdone = done;
        for (int it = 0; it < 64; ++it) {
          if (!__any_sync(0xffffffffu, !fdone)) break;
          const float x = lof + (hif - lof) * fracf;
          const bool ok = !fdone && x > lof && x < hif;
          const bool up = ok && sturm_less_f(ddf, e2f, n, x) > kth;
          float nlo = (ok && !up) ? x : lof;
          float nhi = (ok && up) ? x : hif;
          int any = ok ? 1 : 0;
          for (int o = 1; o < gsz; o <<= 1) {
            nlo = fmaxf(nlo, __shfl_xor_sync(0xffffffffu, nlo, o));
            nhi = fminf(nhi, __shfl_xor_sync(0xffffffffu, nhi, o));
            any |= __shfl_xor_sync(0xffffffffu, any, o);
          }
          if (!fdone) {
            if (!any || !(nlo < nhi)) {
              fdone = true;
            } else {
              lof = nlo;
              hif = nhi;
            }
          }
        }
        lo = fmax(gl, ((double)lof - 4e-6) * tsc);
        hi = fmin(gu, ((double)hif + 4e-6) * tsc);
        // check the widened bracket in FP64: #{λ < lo} <= kth < #{λ < hi}
        int c = 0;
        if (!done) {
          if (gsz >= 2) c = (sl == 0) ? sturm_less(dd, ee2, n, lo, pivmin)
                          : (sl == 1) ? sturm_less(dd, ee2, n, hi, pivmin) : 0;
          else c = sturm_less(dd, ee2, n, lo, pivmin);
        }
        const int base = (lane & ~(gsz - 1));
        const int cl = (gsz >= 2) ? __shfl_sync(0xffffffffu, c, base) : c;
        int ch = (gsz >= 2) ? __shfl_sync(0xffffffffu, c, base + 1) : 0;
        if (gsz < 2 && !done) ch = sturm_less(dd, ee2, n, hi, pivmin);
        if (!done && !(cl <= kth && ch > kth)) {
          lo = gl;
          hi = gu;
        }
      }
      const double tol = 4e-13 * tnorm;
      for (int it = 0; it < 200; ++it) {
        if (!done && !(hi - lo > tol)) done = true;
        if (!__any_sync(0xffffffffu, !done)) break;
        const double x = lo + (hi - lo) * frac;
        const bool ok = !done && x > lo && x < hi;
        const bool up = ok && sturm_less(dd, ee2, n, x, pivmin) > kth;   // eigenvalue below x
        double nlo = (ok && !up) ? x : lo;
        double nhi = (ok && up) ? x : hi;
        int any = ok ? 1 : 0;
        for (int o = 1; o < gsz; o <<= 1) {
          nlo = fmax(nlo, __shfl_xor_sync(0xffffffffu, nlo, o));
          nhi = fmin(nhi, __shfl_xor_sync(0xffffffffu, nhi, o));
          any |= __shfl_xor_sync(0xffffffffu, any, o);
        }
        if (!done) {
          if (!any || !(nlo < nhi)) {
            done = true;
          } else {
            lo = nlo;
            hi = nhi;
          }
        }
      }
      if (e < r && sl == 0) {
        const double lm = 0.5 * (lo + hi);
        lam[e] = lm;
        const double sg = sqrt(fmax(lm, 0.0));
        hv[e] = (sg > beta_d && sg > 0.0) ? (float)((sg - beta_d) / sg) : 0.f;
      }
    }
  }
  __syncthreads();
  if (MODE == 0 && S.nuc) {   // nuclear norm of the patch (src/recon.jl:138-146): Σ σ_i = Σ √λ_i
    const double sq = (tid < r) ? sqrt(fmax(lam[tid], 0.0)) : 0.0;
    const double tot = block_sum_d(sq, redd);
    if (tid == 0) S.nuc[ip] = tot;
    return;
  }
  if (r == 0) {   // (the split stage's back-transform writes the zero columns itself)
    if (MODE == 0)
      for (int64_t q = tid; q < (int64_t)n * n; q += kT) Z[q] = make_float2(0.f, 0.f);
    return;
  }

  // Up to g.rz eigenvectors live in shared memory from here to the output
  // ([row][vector], row stride rz); more use the patch's global slots (row
  // stride n).  zb / zs address them either way.
  const bool stg = r <= g.rz;
  const int64_t zs = stg ? g.rz : n;
  cf* zb = stg ? sY : Z;

  // ---- 3. eigenvectors of T (FP64 twisted factorisation) --------------------
  // z_j in the vector slots read as doubles, D+ after them (shared) or in
  // AUX (global); finally converted in place to complex float.
  if (tid < r) {
    const double lm = lam[tid];
    double* zd = reinterpret_cast<double*>(zb) + tid;
    double* dp = (stg ? reinterpret_cast<double*>(zb) + (int64_t)n * zs : AUX) + tid;
    double q = dd[0] - lm;
    if (fabs(q) < pivmin) q = -pivmin;
    dp[0] = q;
    for (int j = 0; j + 1 < n; ++j) {
      q = dd[j + 1] - lm - ee2[j] / q;
      if (fabs(q) < pivmin) q = -pivmin;
      dp[(int64_t)(j + 1) * zs] = q;
    }
    q = dd[n - 1] - lm;
    if (fabs(q) < pivmin) q = -pivmin;
    zd[(int64_t)(n - 1) * zs] = q;
    int kb = n - 1;
    double gb = fabs(dp[(int64_t)(n - 1) * zs] + q - (dd[n - 1] - lm));
    for (int j = n - 2; j >= 0; --j) {
      q = dd[j] - lm - ee2[j] / q;
      if (fabs(q) < pivmin) q = -pivmin;
      zd[(int64_t)j * zs] = q;
      const double gm = fabs(dp[(int64_t)j * zs] + q - (dd[j] - lm));
      if (gm < gb) {
        gb = gm;
        kb = j;
      }
    }
    double nrm = 1.0, zp = 1.0;
    for (int j = kb - 1; j >= 0; --j) {   // z_j = −e_j z_{j+1} / D+_j
      zp = -ee[j] * zp / dp[(int64_t)j * zs];
      zd[(int64_t)j * zs] = zp;
      nrm += zp * zp;
    }
    zd[(int64_t)kb * zs] = 1.0;
    zp = 1.0;
    for (int j = kb + 1; j < n; ++j) {    // z_j = −e_{j−1} z_{j−1} / D−_j
      zp = -ee[j - 1] * zp / zd[(int64_t)j * zs];
      zd[(int64_t)j * zs] = zp;
      nrm += zp * zp;
    }
    const double inv = 1.0 / sqrt(nrm);
    cf* zc = zb + tid;
    for (int j = 0; j < n; ++j) {
      const double zj = zd[(int64_t)j * zs];
      zc[(int64_t)j * zs] = make_float2((float)(zj * inv), 0.f);
    }
  }
  __syncthreads();
  // Eigenvalues equal to working precision: Gram–Schmidt inside the cluster,
  // cooperatively (every thread walks the same clusters).
  {
    const double ctol = 1e-12 * fmax(tnorm, 1e-300);
    int s0 = 0;
    int rb = 0;
    while (s0 < r) {
      int t = s0 + 1;
      while (t < r && lam[t - 1] - lam[t] <= ctol) ++t;
      for (int qv = s0 + 1; qv < t; ++qv) {
        for (int attempt = 0; attempt < 4; ++attempt) {
          for (int pv = s0; pv < qv; ++pv) {
            double dot = 0.0;
            for (int j = tid; j < n; j += kT) dot += (double)zb[j * zs + pv].x * zb[j * zs + qv].x;
            dot = block_sum_d(dot, redd + 32 * (rb++ & 1));
            for (int j = tid; j < n; j += kT) zb[j * zs + qv].x -= (float)dot * zb[j * zs + pv].x;
            __syncthreads();
          }
          double nr = 0.0;
          for (int j = tid; j < n; j += kT) nr += (double)zb[j * zs + qv].x * zb[j * zs + qv].x;
          nr = sqrt(block_sum_d(nr, redd + 32 * (rb++ & 1)));
          if (nr > 0.1) {
            for (int j = tid; j < n; j += kT) zb[j * zs + qv].x /= (float)nr;
            __syncthreads();
            break;
          }
          // collapsed onto earlier vectors: restart from a unit vector
          for (int j = tid; j < n; j += kT)
            zb[j * zs + qv].x = (j == (qv + attempt * 7919) % n) ? 1.f : 0.f;
          __syncthreads();
        }
      }
      s0 = t;
    }
  }
  if constexpr (MODE == 2) {   // the eigenvalues and √-weights for the back-transform
    double* side = S.side + ip * 6 * (int64_t)n;
    float* sh = reinterpret_cast<float*>(side + 4 * (int64_t)n);
    for (int q = tid; q < r; q += kT) {
      side[3 * n + q] = lam[q];
      sh[q] = hv[q];
    }
    return;
  }

  // ---- 4. V = H_0 ⋯ H_{n-2} Z, blocks of kNb reflectors from the last ---------
  // Staged vectors (few): every thread takes part — S = Yᴴ Z by (output, row
  // group) partial sums added in a fixed order, S ← T S, then Z −= Y S by
  // (row, vector) element, in passes of kCW vectors.  Vectors in global
  // memory (many): thread i updates vector i with its block coefficients in
  // registers.
  // Y: n × kNb, [row][reflector], after the vector stage (16-byte aligned)
  cf* sYb = sY + (((int64_t)n * g.rz + 1) & ~(int64_t)1);
  cf* sT = sYb + (int64_t)n * kNb;    // kNb × kNb, T[a][b] at a*kNb + b
  cf* sYY = sT + kNb * kNb;           // Yᴴ Y
  cf* sS = sYY + kNb * kNb;           // kNb × kCW
  cf* sS2 = sS + kNb * kCW;           // T S
  cf* sP = sS2 + kNb * kCW;           // partial sums, one per thread
  const int nref = n - 1;
  for (int kend = nref; kend > 0; kend -= kNb) {
    const int k0 = max(0, kend - kNb);
    const int nb = kend - k0;
    for (int q = tid; q < n * kNb; q += kT) {   // Y: column jj = reflector k0 + jj
      const int row = q / kNb, jj = q - row * kNb;
      const int k = k0 + jj;
      cf y = make_float2(0.f, 0.f);
      if (jj < nb) {
        if (row == k + 1) y = make_float2(1.f, 0.f);
        else if (row > k + 1) y = A[(int64_t)k * n + row];
      }
      sYb[q] = y;
    }
    __syncthreads();
    if (tid < kNb * kNb) {   // Yᴴ Y
      const int a = tid / kNb, b = tid - a * kNb;
      float sr = 0.f, si = 0.f;
      for (int row = k0 + 1; row < n; ++row) {
        const cf ya = sYb[row * kNb + a], yb = sYb[row * kNb + b];
        sr += ya.x * yb.x + ya.y * yb.y;
        si += ya.x * yb.y - ya.y * yb.x;
      }
      sYY[tid] = make_float2(sr, si);
    }
    __syncthreads();
    if (tid < 32) {   // zlarft (forward, columnwise); lane a owns row a of T
      const int a = tid;
      for (int jj = 0; jj < kNb; ++jj) {
        const cf tj = (jj < nb) ? make_float2(taur[k0 + jj], taui[k0 + jj]) : make_float2(0.f, 0.f);
        if (a < jj) {
          cf sacc = make_float2(0.f, 0.f);
          for (int b = a; b < jj; ++b) sacc = cadd(sacc, cmul(sT[a * kNb + b], sYY[b * kNb + jj]));
          const cf v = cmul(tj, sacc);
          sT[a * kNb + jj] = make_float2(-v.x, -v.y);
        } else if (a < kNb) {
          sT[a * kNb + jj] = (a == jj) ? tj : make_float2(0.f, 0.f);
        }
        __syncwarp();
      }
    }
    __syncthreads();
    if (!stg) {   // vectors in global memory: thread tid updates vector tid (S = Yᴴ z; S ← T S; z −= Y S)
      if (tid < r) bt_vector(Z, n, tid, k0, sYb, sT);
      __syncthreads();
      continue;
    }
    // vectors staged in shared memory: every thread takes part
    for (int c0 = 0; c0 < r; c0 += kCW) {
      const int cw = min(kCW, r - c0);
      const int no = kNb * cw;   // outputs of S = Yᴴ Z (at most 256 <= threads)
      const int ng = kT / no;    // row groups
      if (tid < no * ng) {
        const int o = tid % no, grp = tid / no;
        const int jj = o / cw, c = c0 + (o - jj * cw);
        float sr = 0.f, si = 0.f;
        for (int row = k0 + 1 + grp; row < n; row += ng) {
          const cf y = sYb[row * kNb + jj], z = zb[row * zs + c];   // conj(y)·z
          sr += y.x * z.x + y.y * z.y;
          si += y.x * z.y - y.y * z.x;
        }
        sP[tid] = make_float2(sr, si);
      }
      __syncthreads();
      if (tid < no) {
        float sr = 0.f, si = 0.f;
        for (int gq = 0; gq < ng; ++gq) {
          sr += sP[gq * no + tid].x;
          si += sP[gq * no + tid].y;
        }
        sS[tid] = make_float2(sr, si);
      }
      __syncthreads();
      if (tid < no) {   // T upper-triangular
        const int a = tid / cw, c = tid - a * cw;
        cf sacc = make_float2(0.f, 0.f);
        for (int b = a; b < kNb; ++b) sacc = cadd(sacc, cmul(sT[a * kNb + b], sS[b * cw + c]));
        sS2[tid] = sacc;
      }
      __syncthreads();
      const int rows = n - (k0 + 1);
      for (int q = tid; q < rows * cw; q += kT) {
        const int rr = q / cw, c = q - rr * cw;
        const int row = k0 + 1 + rr;
        cf* zp = zb + row * zs + c0 + c;
        cf z = *zp;
#pragma unroll
        for (int jj = 0; jj < kNb; ++jj) z = csub(z, cmul(sYb[row * kNb + jj], sS2[jj * cw + c]));
        *zp = z;
      }
      __syncthreads();
    }
  }

  // ---- 5. Ṽ = conj(V) diag(√h), columns >= r zero ------------------------------
  if (full) {   // V itself and the eigenvalues
    for (int c = tid; c < n; c += kT) S.lam_out[ip * n + c] = lam[c];
    for (int row = 0; row < n; ++row)
      for (int c = tid; c < n; c += kT) Z[(int64_t)row * n + c] = zb[row * zs + c];
    return;
  }
  for (int row = 0; row < n; ++row) {
    for (int c = tid; c < n; c += kT) {
      cf v = make_float2(0.f, 0.f);
      if (c < r) {
        const cf z = zb[row * zs + c];
        const float sh = sqrtf(hv[c]);
        v = make_float2(z.x * sh, -z.y * sh);
      }
      Z[(int64_t)row * n + c] = v;
    }
  }
}

// ---- split stage, third launch: Ṽ = conj(Q Z) diag(√h) -------------------------
// One CTA per (32 eigenvectors, patch); warp w holds rows w, w + 16, … of its
// 32 vectors in registers (lane = vector) through all WY blocks, taken from
// the last reflector down.  Each block's Y (rows k0+1 … n−1, kYS-strided so a
// row's 16 reflector entries load as warp-wide broadcasts) and T arrive by
// cp.async into one of two buffers while the previous block is applied:
// S = Yᴴ Z by per-warp partial sums added in warp order, S ← T S, then
// Z −= Y S.  The complex products run as packed FP32x2 FMAs on lane-wise
// products, (y.re·z.re, y.im·z.im) and (y.re·z.im, y.im·z.re), combined once
// per row or per reflector.  Columns at or beyond the patch's rank are
// written as zeros.
constexpr int kYS = 18;        // row stride of the staged Y (16-byte aligned rows)
constexpr int kWyThreads = 512;
constexpr int kWyCols = 32;

size_t wy_apply_smem(int nmax) {
  return ((size_t)2 * nmax * kYS + 16 * kNb * kWyCols + 2 * kNb * kWyCols + 2 * kNb * kNb) * sizeof(cf);
}

__device__ __forceinline__ void cpa8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Y rows k0+1 … n−1 of reflectors k0 … k0+nb−1 (the unit entry and the zeros
// above it written directly) and the block's T into (ys, ts); thread t owns
// row k0+1+t (m <= n − 1 < kWyThreads).
__device__ __forceinline__ void wy_stage(const cf* A, int n, int kend, cf* ys, cf* ts, int tid) {
  const int k0 = max(0, kend - kNb), nb = kend - k0;
  const int blk = (n - 1 - kend) / kNb;
  const int m = n - k0 - 1;
  if (tid < m) {
    const int row = k0 + 1 + tid;
    cf* dst = ys + row * kYS;
#pragma unroll
    for (int jj = 0; jj < kNb; ++jj) {
      const int k = k0 + jj;
      if (jj < nb && row > k + 1) cpa8(dst + jj, A + (int64_t)k * n + row);
      else dst[jj] = make_float2((jj < nb && row == k + 1) ? 1.f : 0.f, 0.f);
    }
  }
  if (tid < kNb * kNb) cpa8(ts + tid, A + upper_slot(n, blk * kNb * kNb + tid));
  cpa_commit();
}

template <int RPW>
__global__ void __launch_bounds__(kWyThreads, 1) k_wy_apply(EigArgs g) {
  extern __shared__ __align__(16) unsigned char smraw[];
  int s = 0;
  while (s + 1 < g.nseg && (int64_t)blockIdx.y >= g.seg[s + 1].first) ++s;
  const Seg& S = g.seg[s];
  const int n = S.n;
  const int64_t ip = (int64_t)blockIdx.y - S.first;
  const int cb = blockIdx.x * kWyCols;
  if (cb >= n) return;   // the grid covers the launch's largest n
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const cf* A = S.gram + ip * (int64_t)n * n;
  cf* Z = S.zv + ip * (int64_t)n * n;
  const int r = S.rank[ip];
  const int c = cb + lane;
  if (cb >= r) {
    if (c < n)
      for (int row = w; row < n; row += kWyThreads / 32) Z[(int64_t)row * n + c] = make_float2(0.f, 0.f);
    return;
  }
  const double* side = S.side + ip * 6 * (int64_t)n;
  const float* hw = reinterpret_cast<const float*>(side + 4 * (int64_t)n);
  cf* Ybuf = reinterpret_cast<cf*>(smraw);    // two buffers of n × kYS
  const int ystride = n * kYS;
  cf* part = Ybuf + 2 * ystride;              // 16 warps × kNb × 32
  cf* Ss = part + 16 * kNb * kWyCols;         // kNb × 32
  cf* S2 = Ss + kNb * kWyCols;                // kNb × 32
  cf* Tbuf = S2 + kNb * kWyCols;              // two buffers of kNb × kNb
  float zr[RPW], zi[RPW];
#pragma unroll
  for (int q = 0; q < RPW; ++q) {
    const int row = w + 16 * q;
    zr[q] = (c < r && row < n) ? __ldcg(&Z[(int64_t)row * n + c].x) : 0.f;
    zi[q] = 0.f;
  }
  const int nref = n - 1;
  if (nref > 0) wy_stage(A, n, nref, Ybuf, Tbuf, tid);
  cpa_wait_all();
  __syncthreads();
  int buf = 0;
  for (int kend = nref; kend > 0; kend -= kNb, buf ^= 1) {
    const int k0 = max(0, kend - kNb);
    const cf* Ys = Ybuf + buf * ystride;
    const cf* Ts = Tbuf + buf * kNb * kNb;
    if (kend - kNb > 0)   // the next block, into the other buffers
      wy_stage(A, n, kend - kNb, Ybuf + (buf ^ 1) * ystride, Tbuf + (buf ^ 1) * kNb * kNb, tid);
    // partial S = Yᴴ Z over this warp's rows, eight reflectors per pass
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      unsigned long long P[8], Q[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) P[a] = Q[a] = 0ull;
#pragma unroll
      for (int q = 0; q < RPW; ++q) {
        const int row = w + 16 * q;
        if (row > k0 && row < n) {
          const unsigned long long z1 = pk2(zr[q], zi[q]), z2 = pk2(zi[q], zr[q]);
          const float4* yr = reinterpret_cast<const float4*>(Ys + row * kYS) + 4 * h;
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const float4 y = yr[t];
            const unsigned long long y0 = pk2(y.x, y.y), y1 = pk2(y.z, y.w);
            P[2 * t] = fma2(y0, z1, P[2 * t]);
            Q[2 * t] = fma2(y0, z2, Q[2 * t]);
            P[2 * t + 1] = fma2(y1, z1, P[2 * t + 1]);
            Q[2 * t + 1] = fma2(y1, z2, Q[2 * t + 1]);
          }
        }
      }
#pragma unroll
      for (int a = 0; a < 8; ++a) {   // conj(y)·z = (Σ y.re z.re + y.im z.im, Σ y.re z.im − y.im z.re)
        const float2 p = upk2(P[a]), qq = upk2(Q[a]);
        part[(w * kNb + 8 * h + a) * kWyCols + lane] = make_float2(p.x + p.y, qq.x - qq.y);
      }
    }
    __syncthreads();
    {
      const int a = tid >> 5;   // kWyThreads / 32 = kNb rows of S
      float sr = 0.f, si = 0.f;
#pragma unroll
      for (int w2 = 0; w2 < kWyThreads / 32; ++w2) {
        const cf v = part[(w2 * kNb + a) * kWyCols + lane];
        sr += v.x;
        si += v.y;
      }
      Ss[a * kWyCols + lane] = make_float2(sr, si);
    }
    __syncthreads();
    {
      const int a = tid >> 5;
      cf acc = make_float2(0.f, 0.f);
      for (int b = a; b < kNb; ++b) acc = cadd(acc, cmul(Ts[a * kNb + b], Ss[b * kWyCols + lane]));
      S2[a * kWyCols + lane] = acc;
    }
    __syncthreads();
    // Z −= Y (T S) on this warp's rows, eight reflectors per pass
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      unsigned long long sa[8], sb[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        const cf v = S2[(8 * h + a) * kWyCols + lane];
        sa[a] = pk2(v.x, v.y);
        sb[a] = pk2(v.y, v.x);
      }
#pragma unroll
      for (int q = 0; q < RPW; ++q) {
        const int row = w + 16 * q;
        if (row > k0 && row < n) {
          const float4* yr = reinterpret_cast<const float4*>(Ys + row * kYS) + 4 * h;
          unsigned long long U = 0ull, V = 0ull;
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const float4 y = yr[t];
            const unsigned long long y0 = pk2(y.x, y.y), y1 = pk2(y.z, y.w);
            U = fma2(y0, sa[2 * t], U);
            V = fma2(y0, sb[2 * t], V);
            U = fma2(y1, sa[2 * t + 1], U);
            V = fma2(y1, sb[2 * t + 1], V);
          }
          const float2 u = upk2(U), v = upk2(V);   // y·s = (Σ y.re s.re − y.im s.im, Σ y.re s.im + y.im s.re)
          zr[q] -= u.x - u.y;
          zi[q] -= v.x + v.y;
        }
      }
    }
    cpa_wait_all();
    __syncthreads();
  }
  const float sh = (c < r) ? sqrtf(hw[c]) : 0.f;
#pragma unroll
  for (int q = 0; q < RPW; ++q) {
    const int row = w + 16 * q;
    if (row < n && c < n) Z[(int64_t)row * n + c] = make_float2(zr[q] * sh, -zi[q] * sh);
  }
}

}  // namespace

int eig2_prepare(int nmax) {
  if (nmax > kT) return fail(MSLR_ERR_UNSUPPORTED, "Gram side above 1024");
  if (smem_bytes(nmax, kT, 0) > smem_budget(kT))
    return fail(MSLR_ERR_UNSUPPORTED, "Gram side too large for the eigen stage");
  const int big = (int)smem_budget(kT), small = (int)smem_budget(kSmallT);
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_eig<kT, 1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_eig<kSmallT, 2, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, small));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_eig<kT, 1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_eig<kSmallT, 2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, small));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_eig<kSmallT, kPairsMinB, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(228 * 1024 / kPairsMinB - 1024)));
  const int wy = (int)wy_apply_smem(kSmallT);
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_wy_apply<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, wy));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_wy_apply<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, wy));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_wy_apply<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, wy));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_wy_apply<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, wy));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_wy_apply<20>, cudaFuncAttributeMaxDynamicSharedMemorySize, wy));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_wy_apply<24>, cudaFuncAttributeMaxDynamicSharedMemorySize, wy));
  return MSLR_OK;
}

namespace {

// The split stage applies to thresholded SVSTs (not the values-only or
// all-eigenpairs modes) with a side buffer and 64 <= n <= 384 (the
// back-transform's register tile; the T factors fit the upper triangle).
// MSLR_EIG_SPLIT=0 keeps the one-launch stage everywhere (for comparisons).
bool split_ok(const EigSegment& e) {
  static const bool off = [] {
    const char* v = std::getenv("MSLR_EIG_SPLIT");
    return v && v[0] == '0';
  }();
  if (off || !e.side || e.nuc || e.lam_out || e.n < 64 || e.n > kSmallT) return false;
  const int64_t nblk = (e.n - 1 + kNb - 1) / kNb;
  return nblk * kNb * kNb <= (int64_t)e.n * (e.n - 1) / 2;
}

int wy_apply_launch(const EigArgs& a, int nmax, int64_t total, cudaStream_t st) {
  const dim3 grid((unsigned)((nmax + kWyCols - 1) / kWyCols), (unsigned)total);
  const size_t sm = wy_apply_smem(nmax);
  const int rpw = (nmax + 15) / 16;
  if (rpw <= 4) k_wy_apply<4><<<grid, kWyThreads, sm, st>>>(a);
  else if (rpw <= 8) k_wy_apply<8><<<grid, kWyThreads, sm, st>>>(a);
  else if (rpw <= 12) k_wy_apply<12><<<grid, kWyThreads, sm, st>>>(a);
  else if (rpw <= 16) k_wy_apply<16><<<grid, kWyThreads, sm, st>>>(a);
  else if (rpw <= 20) k_wy_apply<20><<<grid, kWyThreads, sm, st>>>(a);
  else k_wy_apply<24><<<grid, kWyThreads, sm, st>>>(a);
  return MSLR_OK;
}

// One launch (or, for the split stage, three) over segments that all take the
// same CTA variant.
int eig_launch_group(const std::vector<const EigSegment*>& segs, const double* thr, int thr_per_patch,
                     cudaStream_t st, uint64_t* launches) {
  EigArgs a;
  a.nseg = (int)segs.size();
  a.thr = thr;
  a.thr_per_patch = thr_per_patch;
  int64_t total = 0;
  int nmax = 1;
  bool split = true;
  for (int s = 0; s < a.nseg; ++s) {
    Seg& S = a.seg[s];
    const EigSegment& e = *segs[s];
    S.n = e.n;
    S.first = total;
    S.np = e.np;
    S.gram = e.gram;
    S.zv = e.zv;
    S.aux = e.aux;
    S.rank = e.rank;
    S.lam = e.lam;
    S.nuc = e.nuc;
    S.lam_out = e.lam_out;
    S.side = e.side;
    total += e.np;
    nmax = std::max(nmax, e.n);
    split = split && split_ok(e);
  }
  bool big = nmax > kSmallT;
  for (const EigSegment* e : segs) big = big || e->big;
  const int threads = big ? kT : kSmallT;
  if (split) {
    a.rz = 0;
    const size_t sm1 = vec_bytes(nmax) +
                       std::max(threads <= kSmallT ? part_bytes(nmax) : (size_t)0, wy_bytes(nmax, threads)) + 128;
    if (threads == kSmallT)
      k_eig<kSmallT, 2, 1><<<(unsigned)total, kSmallT, sm1, st>>>(a);
    else
      k_eig<kT, 1, 1><<<(unsigned)total, kT, sm1, st>>>(a);
    k_eig<kSmallT, kPairsMinB, 2><<<(unsigned)total, kSmallT, vec_bytes(nmax) + 128, st>>>(a);
    wy_apply_launch(a, nmax, total, st);
    MSLR_CUDA_TRY(cudaGetLastError());
    if (launches) *launches += 3;
    return MSLR_OK;
  }
  a.rz = stage_cols(nmax, threads);
  const size_t sm = smem_bytes(nmax, threads, a.rz);
  if (threads == kSmallT)
    k_eig<kSmallT, 2, 0><<<(unsigned)total, kSmallT, sm, st>>>(a);
  else
    k_eig<kT, 1, 0><<<(unsigned)total, kT, sm, st>>>(a);
  MSLR_CUDA_TRY(cudaGetLastError());
  if (launches) *launches += 1;
  return MSLR_OK;
}

}  // namespace

// Segments with Gram side <= 384 run in the 384-thread variant (two patches per
// SM), larger ones in the 1024-thread variant: one launch per variant present.
// Per-patch thresholds (thr_per_patch) index patches across all segments, so
// such calls keep every segment in one launch.
int eig_launch_multi(int nseg, const EigSegment* segs, const double* thr, int thr_per_patch,
                     cudaStream_t st, uint64_t* launches) {
  if (nseg < 1 || nseg > kMaxSeg) return fail(MSLR_ERR_UNSUPPORTED, "too many scales in one launch");
  std::vector<const EigSegment*> small, big, all;
  for (int s = 0; s < nseg; ++s) {
    (segs[s].n <= kSmallT && !segs[s].big ? small : big).push_back(&segs[s]);
    all.push_back(&segs[s]);
  }
  if (thr_per_patch || small.empty() || big.empty())
    return eig_launch_group(all, thr, thr_per_patch, st, launches);
  int rc = eig_launch_group(big, thr, 0, st, launches);
  if (!rc) rc = eig_launch_group(small, thr, 0, st, launches);
  return rc;
}

int eig2_launch(int n, int64_t np, cf* gram, cf* zv, float* aux, int* rank, const double* thr,
                int thr_per_patch, double lam, cudaStream_t st, int big, double* side, uint64_t* launches) {
  EigSegment s;
  s.n = n;
  s.np = np;
  s.gram = gram;
  s.zv = zv;
  s.aux = reinterpret_cast<double*>(aux);
  s.rank = rank;
  s.lam = lam;
  s.big = big;
  s.nuc = nullptr;
  s.side = side;
  return eig_launch_multi(1, &s, thr, thr_per_patch, st, launches);
}

}  // namespace mslr
