// gram_mma.cu — patch Gram matrices and rebuilds on the tensor cores (tuned form).
//
// Both products are complex GEMMs C = A Bᵀ whose operands are rows with the
// contraction index K contiguous, computed as real GEMMs over 2K with each
// complex value interleaved as (re, im) along K:
//   Re C = Σ_K A[r][K] B[c][K],   Im C = Σ_K A'[r][K] B[c][K],
// where A' is A multiplied by −i (Gram) or +i (rebuild) — for an interleaved
// pair that is a swap of the halves and one sign flip, exact in any precision.
//   Gram     G = M Mᴴ:  A = B = rows of M (K = L), A' = −i·A, C = G
//   rebuild  M_out = W M: A = conj(W) rows (K = n; W is Hermitian, so this is
//            a column of the stored W), B = columns of M, A' = +i·A
// with M = Pᴴ for tall patches (p >= Nt) and M = P otherwise (see svst.cu).
//
// Split precision: every FP32 value v is carried as hi = bf16(v) and
// lo = bf16(v − hi), and each product is hi·hi + hi·lo + lo·hi with FP32
// accumulation (the dropped lo·lo term is ~2^-16 relative).
//
// Kernel structure (mma.sync m16n8k16, BF16 in, FP32 accumulate): one CTA of
// 8 warps computes a 128 × 128 output tile; each warp owns 64 × 32.  K is
// consumed 32 complex values at a time: the FP32 tile pair is gathered into
// shared memory with cp.async (zero-filled outside the matrix), converted
// once into BF16 hi/lo tiles (and the rotated A'), and the gather of the next
// chunk is in flight while the tensor cores work on the current one.  Patch
// element addresses come from per-row and per-K offset tables built once per
// tile / chunk, so the gather does no index arithmetic per element.
#include <cuda_bf16.h>

#include <mutex>

#include "internal.h"
#include "patchmap.cuh"

namespace mslr {

namespace {

constexpr int kBM = 128;       // output tile rows
constexpr int kBN = 128;       // output tile columns
constexpr int kKC = 32;        // complex K per chunk
constexpr int kLdR = 33;       // raw FP32 row stride (complex elements; odd: no bank conflicts)
constexpr int kLdB = 36;       // BF16 row stride (32-bit words = complex elements)
constexpr int kThreads = 256;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// split (re, im) into hi and lo BF16 pairs (low half = re)
__device__ __forceinline__ void split2(float re, float im, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(re - hf.x, im - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// (re, im) → (im, −re) = −i·z ;  (re, im) → (−im, re) = +i·z
__device__ __forceinline__ uint32_t mul_minus_i(uint32_t v) {
  return ((v >> 16) | (v << 16)) ^ 0x80000000u;
}
__device__ __forceinline__ uint32_t mul_plus_i(uint32_t v) {
  return ((v >> 16) | (v << 16)) ^ 0x00008000u;
}

// Not volatile: the scheduler may interleave independent products.
__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b) {
  asm(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Shared memory of one CTA.
struct Smem {
  cf rawA[kBM * kLdR];
  cf rawB[kBN * kLdR];
  uint32_t ah[kBM * kLdB], al[kBM * kLdB];   // A hi / lo
  uint32_t rh[kBM * kLdB], rl[kBM * kLdB];   // rotated A' hi / lo
  uint32_t bh[kBN * kLdB], bl[kBN * kLdB];   // B hi / lo
  int rowA[kBM], rowB[kBN];                  // element offset of each tile row
  int kA[kKC], kB[kKC];                      // element offset of each K of the chunk
};

// Gather chunk (FP32) of rows [0, kBM) × K [0, kKC): element at base + row[r] + kof[kc].
// rows/K outside the matrix (row[r] < 0 or kof[kc] < 0) are zero-filled.  Consecutive
// threads walk K when K is the contiguous axis in memory (kfast), else the rows.
__device__ __forceinline__ void gather(cf* raw, const cf* __restrict__ base, const int* row,
                                       const int* kof, int nrows, bool kfast) {
  for (int q = threadIdx.x; q < nrows * kKC; q += kThreads) {
    int r, kc;
    if (kfast) {
      r = q / kKC;
      kc = q - r * kKC;
    } else {
      kc = q / nrows;
      r = q - kc * nrows;
    }
    const int ro = row[r], ko = kof[kc];
    const bool ok = (ro >= 0) && (ko >= 0);
    cp_async8(raw + r * kLdR + kc, base + (ok ? (int64_t)ro + ko : 0), ok);
  }
}

// FP32 tile → BF16 hi/lo (optionally conjugated), plus the rotated copy.
template <int ROT>   // 0: no rotated copy, -1: −i, +1: +i
__device__ __forceinline__ void convert(const cf* raw, uint32_t* hi, uint32_t* lo, uint32_t* rhi,
                                        uint32_t* rlo, int nrows, bool conj) {
  for (int q = threadIdx.x; q < nrows * kKC; q += kThreads) {
    const int r = q / kKC, kc = q - r * kKC;
    cf v = raw[r * kLdR + kc];
    if (conj) v.y = -v.y;
    uint32_t h, l;
    split2(v.x, v.y, h, l);
    hi[r * kLdB + kc] = h;
    lo[r * kLdB + kc] = l;
    if (ROT == -1) {
      rhi[r * kLdB + kc] = mul_minus_i(h);
      rlo[r * kLdB + kc] = mul_minus_i(l);
    } else if (ROT == 1) {
      rhi[r * kLdB + kc] = mul_plus_i(h);
      rlo[r * kLdB + kc] = mul_plus_i(l);
    }
  }
}

// Four 8×8 b16 matrices from shared memory; lane l supplies the row address of
// matrix l/8 and receives, in register i, the pair (row l/4, cols 2(l%4)..+1) of
// matrix i — for one 32-bit word per complex value that is word (l/4, l%4).
__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const uint32_t* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}

// One chunk of MMAs: warp (wm, wn) accumulates its 64 × 32 quadrant.  A operand
// fragment (m16 × k16): words (g, t), (g+8, t), (g, t+4), (g+8, t+4); B fragment
// (k16 × n8): words (g, t), (g, t+4) of the B rows, g = lane/4, t = lane%4.
__device__ __forceinline__ void mma_chunk(const Smem& s, const uint32_t* bh, const uint32_t* bl,
                                          float (&cr)[4][4][4], float (&ci)[4][4][4]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 2, wn = warp & 3;
  // ldmatrix source rows: A — matrices (rows +0, k +0), (+8, +0), (+0, +4), (+8, +4);
  //                       B — (rows +0, k +0), (+0, +4), (+8, +0), (+8, +4) for two n8 blocks
  const int a_row = wm * 64 + (lane & 7) + ((lane >> 3) & 1) * 8, a_kw = (lane >> 4) * 4;
  const int b_row = wn * 32 + (lane & 7) + (lane >> 4) * 8, b_kw = ((lane >> 3) & 1) * 4;
#pragma unroll
  for (int ks = 0; ks < kKC / 8; ++ks) {
    uint32_t fbh[4][2], fbl[4][2];
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) {
      const int o = (b_row + jj * 16) * kLdB + ks * 8 + b_kw;
      uint32_t t[4];
      ldsm_x4(t, bh + o);
      fbh[2 * jj][0] = t[0];
      fbh[2 * jj][1] = t[1];
      fbh[2 * jj + 1][0] = t[2];
      fbh[2 * jj + 1][1] = t[3];
      ldsm_x4(t, bl + o);
      fbl[2 * jj][0] = t[0];
      fbl[2 * jj][1] = t[1];
      fbl[2 * jj + 1][0] = t[2];
      fbl[2 * jj + 1][1] = t[3];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int o = (a_row + i * 16) * kLdB + ks * 8 + a_kw;
      uint32_t fah[4], fal[4], frh[4], frl[4];
      ldsm_x4(fah, s.ah + o);
      ldsm_x4(fal, s.al + o);
      ldsm_x4(frh, s.rh + o);
      ldsm_x4(frl, s.rl + o);
      // the three split products of an accumulator are 8 MMAs apart, so no
      // MMA waits on the one before it
#pragma unroll
      for (int j = 0; j < 4; ++j) mma_bf16(cr[i][j], fah, fbh[j]);
#pragma unroll
      for (int j = 0; j < 4; ++j) mma_bf16(ci[i][j], frh, fbh[j]);
#pragma unroll
      for (int j = 0; j < 4; ++j) mma_bf16(cr[i][j], fah, fbl[j]);
#pragma unroll
      for (int j = 0; j < 4; ++j) mma_bf16(ci[i][j], frh, fbl[j]);
#pragma unroll
      for (int j = 0; j < 4; ++j) mma_bf16(cr[i][j], fal, fbh[j]);
#pragma unroll
      for (int j = 0; j < 4; ++j) mma_bf16(ci[i][j], frl, fbh[j]);
    }
  }
}

__device__ __forceinline__ void zero_acc(float (&cr)[4][4][4], float (&ci)[4][4][4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) cr[i][j][q] = ci[i][j][q] = 0.f;
}

// ---------------------------------------------------------------------------
// Gram: grid (ntri, Np, nsplit); tile pair (ta >= tb) of the lower triangle,
// K range [split·lchunk, (split+1)·lchunk).  Output column-major G[b·n + a]
// (split partials into out + split·n²), mirrored for off-diagonal tiles.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1)
    k_gram_tc(const cf* __restrict__ img, PatchMap m, cf* __restrict__ out, int nsplit,
              int lchunk) {
  extern __shared__ __align__(16) unsigned char smraw[];
  Smem& s = *reinterpret_cast<Smem*>(smraw);
  int t = blockIdx.x, ta = 0;
  while (t > ta) {
    t -= ta + 1;
    ++ta;
  }
  const int tb = t;
  const bool diag = (ta == tb);
  const int64_t ip = blockIdx.y;
  const int split = blockIdx.z;
  const int64_t org = patch_origin(m, ip);
  const int64_t ts = tstride(m);
  const int a0 = ta * kBM, b0 = tb * kBN;
  const int l_begin = split * lchunk;
  const int l_end = min(m.L, l_begin + lchunk);
  const int n = m.n;
  // row offsets: M[a][l] = (tall) conj(img[a·ts + org + off(l)]) or img[l·ts + org + off(a)]
  for (int r = threadIdx.x; r < kBM; r += kThreads) {
    const int a = a0 + r, b = b0 + r;
    s.rowA[r] = (a < n) ? (int)(m.tall ? (int64_t)a * ts : patch_off(m, a)) : -1;
    s.rowB[r] = (b < n) ? (int)(m.tall ? (int64_t)b * ts : patch_off(m, b)) : -1;
  }
  auto kofs = [&](int l0) {
    if (threadIdx.x < kKC) {
      const int l = l0 + threadIdx.x;
      const int v = (l < l_end) ? (int)(m.tall ? patch_off(m, l) : (int64_t)l * ts) : -1;
      s.kA[threadIdx.x] = v;
      s.kB[threadIdx.x] = v;
    }
  };
  const cf* base = img + org;
  const bool kfast = m.tall != 0;   // tall: K runs over voxels (x-contiguous); wide: over frames
  float cr[4][4][4], ci[4][4][4];
  zero_acc(cr, ci);
  kofs(l_begin);
  __syncthreads();
  if (l_begin < l_end) {
    gather(s.rawA, base, s.rowA, s.kA, kBM, kfast);
    if (!diag) gather(s.rawB, base, s.rowB, s.kB, kBN, kfast);
  }
  cp_commit();
  for (int l0 = l_begin; l0 < l_end; l0 += kKC) {
    cp_wait_all();
    __syncthreads();   // raw chunk landed; previous MMAs done with the BF16 tiles
    convert<-1>(s.rawA, s.ah, s.al, s.rh, s.rl, kBM, m.tall != 0);
    if (!diag) convert<0>(s.rawB, s.bh, s.bl, nullptr, nullptr, kBN, m.tall != 0);
    __syncthreads();   // raw buffers free, K offsets of this chunk consumed
    const int l1 = l0 + kKC;
    if (l1 < l_end) {
      kofs(l1);
      __syncthreads();
      gather(s.rawA, base, s.rowA, s.kA, kBM, kfast);
      if (!diag) gather(s.rawB, base, s.rowB, s.kB, kBN, kfast);
    }
    cp_commit();
    mma_chunk(s, diag ? s.ah : s.bh, diag ? s.al : s.bl, cr, ci);
  }
  cf* G = out + ((nsplit > 1) ? (int64_t)split * n * n : ip * (int64_t)n * n);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 2, wn = warp & 3;
  const int g = lane >> 2, tig = lane & 3;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int a = a0 + wm * 64 + i * 16 + g + h * 8;
          const int b = b0 + wn * 32 + j * 8 + tig * 2 + q;
          if (a < n && b < n) {
            const cf v = make_float2(cr[i][j][h * 2 + q], ci[i][j][h * 2 + q]);
            G[(int64_t)b * n + a] = v;
            if (!diag) G[(int64_t)a * n + b] = cconj(v);
          }
        }
}

// ---------------------------------------------------------------------------
// Rebuild: grid (ceil(n/128), ceil(L/128), Np).  A rows a: conj(W[a][·]) =
// stored W column a; B rows l: M[·][l].  Tall patches write conj(M_out[a][l])
// to frame a, voxel l; wide patches M_out[a][l] to frame l, voxel a; into the
// image (exact partitions) or the per-patch buffer (p, Nt, Np).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1)
    k_rebuild_tc(const cf* __restrict__ img, const cf* __restrict__ W, PatchMap m,
                 cf* __restrict__ out, int direct) {
  extern __shared__ __align__(16) unsigned char smraw[];
  Smem& s = *reinterpret_cast<Smem*>(smraw);
  const int a0 = blockIdx.x * kBM, l0 = blockIdx.y * kBN;
  const int64_t ip = blockIdx.z;
  const int n = m.n;
  const cf* Wp = W + ip * (int64_t)n * n;
  const int64_t org = patch_origin(m, ip);
  const int64_t ts = tstride(m);
  for (int r = threadIdx.x; r < kBM; r += kThreads) {
    const int a = a0 + r, l = l0 + r;
    s.rowA[r] = (a < n) ? a * n : -1;
    // M[b][l]: tall conj(img[b·ts + org + off(l)]); wide img[l·ts + org + off(b)]
    s.rowB[r] = (l < m.L) ? (int)(m.tall ? patch_off(m, l) : (int64_t)l * ts) : -1;
  }
  auto kofs = [&](int b0) {
    if (threadIdx.x < kKC) {
      const int b = b0 + threadIdx.x;
      s.kA[threadIdx.x] = (b < n) ? b : -1;
      s.kB[threadIdx.x] = (b < n) ? (int)(m.tall ? (int64_t)b * ts : patch_off(m, b)) : -1;
    }
  };
  const cf* bbase = img + org;
  const bool bfast = m.tall == 0;   // B rows: tall → voxels, K frames; wide → frames, K voxels
  float cr[4][4][4], ci[4][4][4];
  zero_acc(cr, ci);
  kofs(0);
  __syncthreads();
  gather(s.rawA, Wp, s.rowA, s.kA, kBM, true);
  gather(s.rawB, bbase, s.rowB, s.kB, kBN, bfast);
  cp_commit();
  for (int b0 = 0; b0 < n; b0 += kKC) {
    cp_wait_all();
    __syncthreads();
    convert<1>(s.rawA, s.ah, s.al, s.rh, s.rl, kBM, false);
    convert<0>(s.rawB, s.bh, s.bl, nullptr, nullptr, kBN, m.tall != 0);
    __syncthreads();
    const int b1 = b0 + kKC;
    if (b1 < n) {
      kofs(b1);
      __syncthreads();
      gather(s.rawA, Wp, s.rowA, s.kA, kBM, true);
      gather(s.rawB, bbase, s.rowB, s.kB, kBN, bfast);
    }
    cp_commit();
    mma_chunk(s, s.bh, s.bl, cr, ci);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 2, wn = warp & 3;
  const int g = lane >> 2, tig = lane & 3;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int a = a0 + wm * 64 + i * 16 + g + h * 8;
          const int l = l0 + wn * 32 + j * 8 + tig * 2 + q;
          if (a >= n || l >= m.L) continue;
          const float re = cr[i][j][h * 2 + q], im = ci[i][j][h * 2 + q];
          const int pv = m.tall ? l : a;   // voxel within the patch
          const int tt = m.tall ? a : l;   // frame
          const cf v = m.tall ? make_float2(re, -im) : make_float2(re, im);
          if (direct) out[org + patch_off(m, pv) + (int64_t)tt * ts] = v;
          else out[(ip * m.Nt + tt) * (int64_t)m.p + pv] = v;
        }
}

}  // namespace

// Dynamic shared memory above 48 KB is opted into once per device.
int tc_prepare() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  MSLR_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 64 && done[dev]) return MSLR_OK;
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(Smem)));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_rebuild_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(Smem)));
  if (dev < 64) done[dev] = true;
  return MSLR_OK;
}

// Offsets are kept in 32-bit tables: every element must lie within 2^31
// elements of its patch origin, and n² below 2^31.
bool mma_supported(const PatchMap& m) {
  const int64_t span = m.batch ? m.mstride : (int64_t)m.Nt * m.nvox;
  return span < (int64_t)0x7fffffff && (int64_t)m.n * m.n < (int64_t)0x7fffffff;
}

int gram_mma_launch(const cf* img, const PatchMap& m, int64_t np, cf* out_or_part, int nsplit,
                    int lchunk, cudaStream_t st) {
  if (int rc = tc_prepare()) return rc;
  const int T = (m.n + kBM - 1) / kBM;
  const int ntri = T * (T + 1) / 2;
  k_gram_tc<<<dim3(ntri, (unsigned)np, nsplit), kThreads, sizeof(Smem), st>>>(img, m, out_or_part,
                                                                              nsplit, lchunk);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int rebuild_mma_launch(const cf* img, const cf* W, const PatchMap& m, int64_t np, cf* out,
                       int direct, cudaStream_t st) {
  if (int rc = tc_prepare()) return rc;
  k_rebuild_tc<<<dim3((m.n + kBM - 1) / kBM, (m.L + kBN - 1) / kBN, (unsigned)np), kThreads,
                 sizeof(Smem), st>>>(img, W, m, out, direct);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

}  // namespace mslr
