// gram_mma.cu — patch Gram matrices on the tensor cores (tuned form).
//
// G = M Mᴴ for every patch (M = Pᴴ when p >= Nt, else P; see svst.cu), as a
// real GEMM over K = 2L with the complex values interleaved along K:
//   Gr[a][b] = Σ_K A[a][K] B[b][K],   A = B = (Re M, Im M) interleaved,
//   Gi[a][b] = Σ_K A'[a][K] B[b][K],  A' = (Im M, −Re M) = −i·M interleaved,
// so both operands are rows of the same K-major tile and A' is the A tile
// with each (re, im) pair swapped and one half negated (exact, in registers).
// Split precision: each FP32 value v is carried as hi = bf16(v) and
// lo = bf16(v − hi); every product is hi·hi + hi·lo + lo·hi with FP32
// accumulation (the dropped lo·lo term is ~2^-16 relative).
//
// mma.sync.m16n8k16 (BF16 in, FP32 accumulate).  CTA = 4 warps, one 64×64
// output tile of the lower triangle (patch, tile pair, K split) per CTA; each
// warp owns a 32×32 quadrant (2 m16 × 4 n8 fragments for Gr and for Gi).
// K is staged 32 complex values (64 real K) at a time through shared memory.
#include <cuda_bf16.h>

#include "internal.h"
#include "patchmap.cuh"

namespace mslr {

namespace {

constexpr int kTM = 64;        // output tile side
constexpr int kKC = 32;        // complex K values per stage
constexpr int kLd = 36;        // shared row stride in 32-bit words (bank-conflict-free fragments)
constexpr int kThreads = 128;

__device__ __forceinline__ uint32_t pack_bf16(float lo_half, float hi_half) {
  // low 16 bits = first element (K even = real part), high 16 bits = second
  __nv_bfloat162 v = __floats2bfloat162_rn(lo_half, hi_half);
  return *reinterpret_cast<uint32_t*>(&v);
}

// split (re, im) into hi and lo bf16 pairs
__device__ __forceinline__ void split2(float re, float im, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat16 hr = __float2bfloat16_rn(re), hi_ = __float2bfloat16_rn(im);
  const float rr = re - __bfloat162float(hr), ri = im - __bfloat162float(hi_);
  __nv_bfloat162 h;
  h.x = hr;
  h.y = hi_;
  hi = *reinterpret_cast<uint32_t*>(&h);
  lo = pack_bf16(rr, ri);
}

// (re, im) → (im, −re): multiply the interleaved pair by −i
__device__ __forceinline__ uint32_t mul_minus_i(uint32_t v) {
  const uint32_t swapped = (v >> 16) | (v << 16);   // (im, re)
  return swapped ^ 0x80000000u;                      // (im, −re)
}

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

}  // namespace

__global__ void __launch_bounds__(kThreads) k_gram_mma(const cf* __restrict__ img, PatchMap m,
                                                       cf* __restrict__ out, int nsplit,
                                                       int lchunk) {
  __shared__ uint32_t sAh[kTM * kLd], sAl[kTM * kLd], sBh[kTM * kLd], sBl[kTM * kLd];
  int t = blockIdx.x, ta = 0;
  while (t > ta) {
    t -= ta + 1;
    ++ta;
  }
  const int tb = t;
  const int64_t ip = blockIdx.y;
  const int split = blockIdx.z;
  const int64_t org = patch_origin(m, ip);
  const int a0 = ta * kTM, b0 = tb * kTM;
  const int l_begin = split * lchunk;
  const int l_end = min(m.L, l_begin + lchunk);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wa = warp >> 1, wb = warp & 1;   // 2 × 2 warps of 32 × 32
  const int g = lane >> 2, tig = lane & 3;
  float cr[2][4][4], ci[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) cr[i][j][q] = ci[i][j][q] = 0.f;

  for (int l0 = l_begin; l0 < l_end; l0 += kKC) {
    // stage A (rows a0..) and B (rows b0..) for complex K l0..l0+31
    for (int q = threadIdx.x; q < kTM * kKC; q += kThreads) {
      int r, kc;
      if (m.tall) {   // consecutive threads along l (voxel-contiguous)
        kc = q % kKC;
        r = q / kKC;
      } else {        // consecutive threads along the voxel row index
        r = q % kTM;
        kc = q / kTM;
      }
      const int l = l0 + kc;
      cf va = make_float2(0.f, 0.f), vb = make_float2(0.f, 0.f);
      if (l < l_end) {
        if (a0 + r < m.n) va = m_elem(m, img, org, a0 + r, l);
        if (b0 + r < m.n) vb = (ta == tb) ? va : m_elem(m, img, org, b0 + r, l);
      }
      uint32_t h, lo;
      split2(va.x, va.y, h, lo);
      sAh[r * kLd + kc] = h;
      sAl[r * kLd + kc] = lo;
      split2(vb.x, vb.y, h, lo);
      sBh[r * kLd + kc] = h;
      sBl[r * kLd + kc] = lo;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < kKC / 8; ++ks) {   // 8 complex = 16 real K per mma
      const int kc0 = ks * 8;
      uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r0 = wa * 32 + i * 16 + g;
        ah[i][0] = sAh[r0 * kLd + kc0 + tig];
        ah[i][1] = sAh[(r0 + 8) * kLd + kc0 + tig];
        ah[i][2] = sAh[r0 * kLd + kc0 + tig + 4];
        ah[i][3] = sAh[(r0 + 8) * kLd + kc0 + tig + 4];
        al[i][0] = sAl[r0 * kLd + kc0 + tig];
        al[i][1] = sAl[(r0 + 8) * kLd + kc0 + tig];
        al[i][2] = sAl[r0 * kLd + kc0 + tig + 4];
        al[i][3] = sAl[(r0 + 8) * kLd + kc0 + tig + 4];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c0 = wb * 32 + j * 8 + g;
        bh[j][0] = sBh[c0 * kLd + kc0 + tig];
        bh[j][1] = sBh[c0 * kLd + kc0 + tig + 4];
        bl[j][0] = sBl[c0 * kLd + kc0 + tig];
        bl[j][1] = sBl[c0 * kLd + kc0 + tig + 4];
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        uint32_t aih[4], ail[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          aih[q] = mul_minus_i(ah[i][q]);
          ail[q] = mul_minus_i(al[i][q]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          mma_bf16(cr[i][j], ah[i], bh[j]);
          mma_bf16(cr[i][j], ah[i], bl[j]);
          mma_bf16(cr[i][j], al[i], bh[j]);
          mma_bf16(ci[i][j], aih, bh[j]);
          mma_bf16(ci[i][j], aih, bl[j]);
          mma_bf16(ci[i][j], ail, bh[j]);
        }
      }
    }
    __syncthreads();
  }
  const int n = m.n;
  cf* G = out + ((nsplit > 1) ? (int64_t)split * n * n : ip * (int64_t)n * n);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int a = a0 + wa * 32 + i * 16 + g + h * 8;
          const int b = b0 + wb * 32 + j * 8 + tig * 2 + q;
          if (a < n && b < n) {
            const cf v = make_float2(cr[i][j][h * 2 + q], ci[i][j][h * 2 + q]);
            G[(int64_t)b * n + a] = v;
            if (ta != tb) G[(int64_t)a * n + b] = cconj(v);
          }
        }
}

// ---------------------------------------------------------------------------
// Rebuild M_out = W M on the tensor cores, as a real GEMM over K = 2n with
// (b, re/im) interleaved:
//   Re M_out[a][l] = Σ_K A[a][K]  B[l][K],  A  = conj(W[a][·]) interleaved
//   Im M_out[a][l] = Σ_K A'[a][K] B[l][K],  A' = i·A (pair swapped, one half negated)
//   B[l][(b, ·)] = M[b][l] interleaved.
// W is Hermitian, so row a of conj(W) is column a of W — contiguous in the
// column-major storage.  Output: tall patches write conj(M_out[a][l]) to
// frame a, voxel l; wide patches M_out[a][l] to frame l, voxel a; either into
// the image (exact partitions) or the per-patch buffer (p, Nt, Np).
// grid (ceil(n/64), ceil(L/64), Np).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t mul_plus_i(uint32_t v) {
  const uint32_t swapped = (v >> 16) | (v << 16);   // (im, re)
  return swapped ^ 0x00008000u;                      // (−im, re)
}

__global__ void __launch_bounds__(kThreads) k_rebuild_mma(const cf* __restrict__ img,
                                                          const cf* __restrict__ W, PatchMap m,
                                                          cf* __restrict__ out, int direct) {
  __shared__ uint32_t sAh[kTM * kLd], sAl[kTM * kLd], sBh[kTM * kLd], sBl[kTM * kLd];
  const int a0 = blockIdx.x * kTM, l0 = blockIdx.y * kTM;
  const int64_t ip = blockIdx.z;
  const int n = m.n;
  const cf* Wp = W + ip * (int64_t)n * n;
  const int64_t org = patch_origin(m, ip);
  const int64_t ts = tstride(m);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wa = warp >> 1, wb = warp & 1;
  const int g = lane >> 2, tig = lane & 3;
  float cr[2][4][4], ci[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) cr[i][j][q] = ci[i][j][q] = 0.f;

  for (int b0 = 0; b0 < n; b0 += kKC) {
    for (int q = threadIdx.x; q < kTM * kKC; q += kThreads) {
      {   // A: conj(W[a][b]) = W[b][a], stored at a*n + b (contiguous in b)
        const int kc = q % kKC, r = q / kKC;
        const int a = a0 + r, b = b0 + kc;
        cf w = make_float2(0.f, 0.f);
        if (a < n && b < n) w = Wp[(int64_t)a * n + b];
        uint32_t h, lo;
        split2(w.x, w.y, h, lo);
        sAh[r * kLd + kc] = h;
        sAl[r * kLd + kc] = lo;
      }
      {   // B: row l, K = b: M[b][l]
        int r, kc;
        if (m.tall) {   // M[b][l] = conj(img[b][vox_l]): consecutive threads along l
          r = q % kTM;
          kc = q / kTM;
        } else {        // M[b][l] = img[l][vox_b]: consecutive threads along b
          kc = q % kKC;
          r = q / kKC;
        }
        const int l = l0 + r, b = b0 + kc;
        cf v = make_float2(0.f, 0.f);
        if (l < m.L && b < n) v = m_elem(m, img, org, b, l);
        uint32_t h, lo;
        split2(v.x, v.y, h, lo);
        sBh[r * kLd + kc] = h;
        sBl[r * kLd + kc] = lo;
      }
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < kKC / 8; ++ks) {
      const int kc0 = ks * 8;
      uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r0 = wa * 32 + i * 16 + g;
        ah[i][0] = sAh[r0 * kLd + kc0 + tig];
        ah[i][1] = sAh[(r0 + 8) * kLd + kc0 + tig];
        ah[i][2] = sAh[r0 * kLd + kc0 + tig + 4];
        ah[i][3] = sAh[(r0 + 8) * kLd + kc0 + tig + 4];
        al[i][0] = sAl[r0 * kLd + kc0 + tig];
        al[i][1] = sAl[(r0 + 8) * kLd + kc0 + tig];
        al[i][2] = sAl[r0 * kLd + kc0 + tig + 4];
        al[i][3] = sAl[(r0 + 8) * kLd + kc0 + tig + 4];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c0 = wb * 32 + j * 8 + g;
        bh[j][0] = sBh[c0 * kLd + kc0 + tig];
        bh[j][1] = sBh[c0 * kLd + kc0 + tig + 4];
        bl[j][0] = sBl[c0 * kLd + kc0 + tig];
        bl[j][1] = sBl[c0 * kLd + kc0 + tig + 4];
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        uint32_t aih[4], ail[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          aih[q] = mul_plus_i(ah[i][q]);
          ail[q] = mul_plus_i(al[i][q]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          mma_bf16(cr[i][j], ah[i], bh[j]);
          mma_bf16(cr[i][j], ah[i], bl[j]);
          mma_bf16(cr[i][j], al[i], bh[j]);
          mma_bf16(ci[i][j], aih, bh[j]);
          mma_bf16(ci[i][j], aih, bl[j]);
          mma_bf16(ci[i][j], ail, bh[j]);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int a = a0 + wa * 32 + i * 16 + g + h * 8;
          const int l = l0 + wb * 32 + j * 8 + tig * 2 + q;
          if (a >= n || l >= m.L) continue;
          const float re = cr[i][j][h * 2 + q], im = ci[i][j][h * 2 + q];
          const int pv = m.tall ? l : a;   // voxel within the patch
          const int tt = m.tall ? a : l;   // frame
          const cf v = m.tall ? make_float2(re, -im) : make_float2(re, im);
          if (direct) out[org + patch_off(m, pv) + (int64_t)tt * ts] = v;
          else out[(ip * m.Nt + tt) * (int64_t)m.p + pv] = v;
        }
}

int rebuild_mma_launch(const cf* img, const cf* W, const PatchMap& m, int64_t np, cf* out,
                       int direct, cudaStream_t st) {
  k_rebuild_mma<<<dim3((m.n + kTM - 1) / kTM, (m.L + kTM - 1) / kTM, (unsigned)np), kThreads, 0,
                  st>>>(img, W, m, out, direct);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int gram_mma_launch(const cf* img, const PatchMap& m, int64_t np, cf* out_or_part, int nsplit,
                    int lchunk, cudaStream_t st) {
  const int T = (m.n + kTM - 1) / kTM;
  const int ntri = T * (T + 1) / 2;
  k_gram_mma<<<dim3(ntri, (unsigned)np, nsplit), kThreads, 0, st>>>(img, m, out_or_part, nsplit,
                                                                     lchunk);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

}  // namespace mslr
