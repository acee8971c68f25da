// gram_umma.cu — patch Grams and rebuilds on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory) for the tuned form.
//
// Patch Grams and rebuilds as complex GEMMs over rows with the
// contraction index K contiguous:
//   Gram     G[a][b]      = Σ_l M[a][l] conj(M[b][l])      (A = B = rows of M)
//   rebuild  M_out[a][l]  = Σ_b W[a][b] M[b][l]            (A = rows of W, B = columns of M)
// with M = Pᴴ for tall patches (p >= Nt), M = P otherwise.  Complex values are
// split into planar real / imaginary BF16 tiles, each FP32 value v carried as
// hi = bf16(v) and lo = bf16(v − hi); a real product x·y is hi·hi + hi·lo +
// lo·hi with FP32 accumulation.  Per 16-element K step one thread issues 12
// M=128 × N=128 × K=16 MMAs into two accumulators (real, imaginary; 256 TMEM
// columns):
//   Gram     Re += Ar·Brᵀ + Ai·Biᵀ      Im += Ai·Brᵀ − Ar·Biᵀ
//   rebuild  Re += Ar·Brᵀ − Ai·Biᵀ      Im += Ar·Biᵀ + Ai·Brᵀ
// (negation through the instruction descriptor).
//
// The TF32 form runs the same products with TF32 operands (one FP32 plane per
// part, rounded to TF32) and four M=128 × N=128 × K=8 kind::tf32 MMAs per
// 8-element K step: Gram Re += Ar·Brᵀ + Ai·Biᵀ, Im += Ai·Brᵀ − Ar·Biᵀ (the
// rebuild's signs as above).
//
// One CTA of 8 warps per 128 × 128 output tile.  K advances 32 elements per
// chunk: every thread loads its share of the next chunk from global memory
// into registers (patch element addresses from per-row / per-K offset
// tables) while the tensor core works on the current chunk, then converts it
// into the K-major, unswizzled core-matrix layout of a free stage (two stages,
// 8 tiles of 8 KB each).  A stage is reused only after the tcgen05.commit of
// the MMAs that read it has arrived on the stage's mbarrier.  The epilogue
// reads the accumulators with tcgen05.ld (warp w: TMEM lanes 32·(w mod 4),
// columns 64·(w / 4)).  Every wait is bounded (DevWait::polls polls).  On a
// time-out the kernel stops issuing work, thread 0 waits (with the default
// poll count) for the MMAs it has already committed, the output tile is
// written as zeros, the tensor memory is freed and kErrMmaWait is raised in
// the caller's error word.
#include <cuda_bf16.h>

#include <mutex>

#include "internal.h"
#include "patchmap.cuh"

namespace mslr {

namespace {

constexpr int kTM = 128;          // output rows per CTA (TMEM lanes)
constexpr int kTN = 128;          // output columns per CTA
constexpr int kKc = 32;           // K elements per chunk
constexpr int kThr = 256;
constexpr int kTile = kTM * kKc;  // bf16 per planar tile
constexpr int kPairs = kTile / 2 / kThr;   // (k, k+1) pairs per thread per operand: 8
constexpr int kTmemCols = 256;

enum { AR_H, AR_L, AI_H, AI_L, BR_H, BR_L, BI_H, BI_L, NOPS };

struct USmem {
  uint32_t op[2][NOPS][kTile / 2];   // two stages × 8 tiles of 128 × 32 bf16 (as bf16 pairs)
  int rowA[kTM], rowB[kTN];
  int kof[2][kKc];
  uint64_t bar[2];
  uint32_t tmem;
};

__device__ __forceinline__ unsigned su32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// word index of the bf16 pair (r, k..k+1), k even, in a K-major unswizzled tile:
// 8-row × 8-element core matrices of 128 bytes, k-adjacent cores 128 B apart
// (LBO), 8-row groups 512 B apart (SBO)
__device__ __forceinline__ int pair_word(int r, int k) {
  return ((r >> 3) * 4 + (k >> 3)) * 32 + (r & 7) * 4 + ((k & 7) >> 1);
}

// shared-memory matrix descriptor (sm_100 layout): start, LBO = 128 B, SBO = 512 B,
// version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc(const void* p) {
  const uint64_t a = su32(p);
  return ((a >> 4) & 0x3FFFull) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) |
         (1ull << 46);
}

// instruction descriptor: BF16 × BF16 → F32, both K-major, M = 128, N = 128
__host__ __device__ constexpr uint32_t idesc(bool negA) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((negA ? 1u : 0u) << 13) | ((uint32_t)(kTN >> 3) << 17) |
         ((uint32_t)(kTM >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t id, bool acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(a), "l"(b), "r"(id), "r"(acc ? 1u : 0u));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   su32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(su32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int polls) {
  const unsigned a = su32(bar);
  for (int it = 0; it < polls; ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// hi/lo split of two consecutive values into packed bf16 pairs (k in the low half)
__device__ __forceinline__ void split_pair(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// TF32 operands (the TF32 form): one FP32 plane per real / imaginary part,
// each value rounded to TF32 (to nearest, ties away), in K-major unswizzled
// core matrices of 8 rows × 4 values (128 bytes): k-adjacent cores 128 B apart
// (LBO), 8-row groups 1024 B apart (SBO).  A chunk of 32 K values is four
// 8-value MMA steps.  Planes per stage: Ar, Ai, Br, Bi of 4096 words each.
constexpr int kTfPlane = kTile;   // words per TF32 plane (128 rows × 32 values)

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ int tf_word(int r, int k) {
  return ((r >> 3) * 8 + (k >> 2)) * 32 + (r & 7) * 4 + (k & 3);
}
__device__ __forceinline__ uint64_t sdesc_tf(const void* p) {
  const uint64_t a = su32(p);
  return ((a >> 4) & 0x3FFFull) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46);
}
// instruction descriptor: TF32 × TF32 → F32, both K-major, M = 128, N = 128
__host__ __device__ constexpr uint32_t idesc_tf(bool negA) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((negA ? 1u : 0u) << 13) | ((uint32_t)(kTN >> 3) << 17) |
         ((uint32_t)(kTM >> 4) << 24);
}
__device__ __forceinline__ void umma_tf(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t id, bool acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(a), "l"(b), "r"(id), "r"(acc ? 1u : 0u));
}

// Registers of one operand chunk: thread t holds pairs q = t + 256 i, i < 8, of
// the 128 × 32 tile; pair q is (row r, k..k+1) of core c = q / 32.
struct Chunk {
  cf v[kPairs][2];
};

__device__ __forceinline__ void pair_rk(int i, int& r, int& k) {
  const int q = threadIdx.x + kThr * i;
  const int c = q >> 5, w = q & 31;
  r = (c >> 2) * 8 + (w >> 2);
  k = (c & 3) * 8 + (w & 3) * 2;
}

__device__ __forceinline__ void load_chunk(Chunk& ch, const cf* __restrict__ base, const int* row,
                                           const int* kof) {
#pragma unroll
  for (int i = 0; i < kPairs; ++i) {
    int r, k;
    pair_rk(i, r, k);
    const int ro = row[r];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const int ko = kof[k + d];
      ch.v[i][d] = (ro >= 0 && ko >= 0) ? __ldg(base + (int64_t)ro + ko) : make_float2(0.f, 0.f);
    }
  }
}

// chunk → planar hi / lo tiles (re_h, re_l, im_h, im_l), conjugated when conj
__device__ __forceinline__ void store_chunk(const Chunk& ch, uint32_t* rh, uint32_t* rl,
                                            uint32_t* ih, uint32_t* il, bool conj) {
#pragma unroll
  for (int i = 0; i < kPairs; ++i) {
    int r, k;
    pair_rk(i, r, k);
    const int w = pair_word(r, k);
    const cf a = ch.v[i][0], b = ch.v[i][1];
    const float ai = conj ? -a.y : a.y, bi = conj ? -b.y : b.y;
    uint32_t h, l;
    split_pair(a.x, b.x, h, l);
    rh[w] = h;
    rl[w] = l;
    split_pair(ai, bi, h, l);
    ih[w] = h;
    il[w] = l;
  }
}

// One operand chunk into stage `stage` (B operand when isB), conjugated when conj.
template <bool TF>
__device__ __forceinline__ void store_operand(const Chunk& ch, uint32_t* stage, bool isB, bool conj) {
  if constexpr (TF) {
    uint32_t* re = stage + (isB ? 2 : 0) * kTfPlane;
    uint32_t* im = stage + (isB ? 3 : 1) * kTfPlane;
#pragma unroll
    for (int i = 0; i < kPairs; ++i) {
      int r, k;
      pair_rk(i, r, k);
      const int w = tf_word(r, k);
      const cf a = ch.v[i][0], b = ch.v[i][1];
      *reinterpret_cast<uint2*>(re + w) = make_uint2(to_tf32(a.x), to_tf32(b.x));
      *reinterpret_cast<uint2*>(im + w) = make_uint2(to_tf32(conj ? -a.y : a.y), to_tf32(conj ? -b.y : b.y));
    }
  } else {
    const int o = isB ? BR_H : AR_H;
    store_chunk(ch, stage + (o + 0) * (kTile / 2), stage + (o + 1) * (kTile / 2),
                stage + (o + 2) * (kTile / 2), stage + (o + 3) * (kTile / 2), conj);
  }
}

// The 12 MMAs of one 16-element K step t of stage s.
template <bool GRAM>
__device__ __forceinline__ void issue_step(const USmem& s, int st, int t, uint32_t dre, uint32_t dim,
                                           bool acc, bool bSameAsA) {
  const uint32_t* o = &s.op[st][0][0];
  auto A = [&](int k) { return sdesc(o + k * (kTile / 2) + t * 64); };   // +2 cores = 256 B = 64 words
  const int bro = bSameAsA ? AR_H : BR_H;   // B operands: same tiles as A on diagonal Gram tiles
  auto B = [&](int k) { return sdesc(o + (bro + (k - BR_H)) * (kTile / 2) + t * 64); };
  constexpr uint32_t P = idesc(false), N = idesc(true);
  // real part
  umma(dre, A(AR_H), B(BR_H), P, acc);
  umma(dre, A(AR_H), B(BR_L), P, true);
  umma(dre, A(AR_L), B(BR_H), P, true);
  umma(dre, A(AI_H), B(BI_H), GRAM ? P : N, true);
  umma(dre, A(AI_H), B(BI_L), GRAM ? P : N, true);
  umma(dre, A(AI_L), B(BI_H), GRAM ? P : N, true);
  // imaginary part
  if (GRAM) {
    umma(dim, A(AI_H), B(BR_H), P, acc);
    umma(dim, A(AI_H), B(BR_L), P, true);
    umma(dim, A(AI_L), B(BR_H), P, true);
    umma(dim, A(AR_H), B(BI_H), N, true);
    umma(dim, A(AR_H), B(BI_L), N, true);
    umma(dim, A(AR_L), B(BI_H), N, true);
  } else {
    umma(dim, A(AR_H), B(BI_H), P, acc);
    umma(dim, A(AR_H), B(BI_L), P, true);
    umma(dim, A(AR_L), B(BI_H), P, true);
    umma(dim, A(AI_H), B(BR_H), P, true);
    umma(dim, A(AI_H), B(BR_L), P, true);
    umma(dim, A(AI_L), B(BR_H), P, true);
  }
}

// All MMAs of the chunk in stage st (first: the accumulators start from zero).
template <bool GRAM, bool TF>
__device__ __forceinline__ void issue_chunk(const USmem& s, int st, uint32_t dre, uint32_t dim,
                                            bool first, bool bSameAsA) {
  if constexpr (TF) {
    const uint32_t* o = &s.op[st][0][0];
    const int br = bSameAsA ? 0 : 2, bi = bSameAsA ? 1 : 3;
    constexpr uint32_t P = idesc_tf(false), N = idesc_tf(true);
#pragma unroll
    for (int t = 0; t < kKc / 8; ++t) {
      auto D = [&](int pl) { return sdesc_tf(o + pl * kTfPlane + t * 64); };   // +2 cores = 256 B
      const bool acc = !first || t > 0;
      // Gram:    Re += Ar·Brᵀ + Ai·Biᵀ   Im += Ai·Brᵀ − Ar·Biᵀ
      // rebuild: Re += Ar·Brᵀ − Ai·Biᵀ   Im += Ar·Biᵀ + Ai·Brᵀ
      umma_tf(dre, D(0), D(br), P, acc);
      umma_tf(dre, D(1), D(bi), GRAM ? P : N, true);
      if (GRAM) {
        umma_tf(dim, D(1), D(br), P, acc);
        umma_tf(dim, D(0), D(bi), N, true);
      } else {
        umma_tf(dim, D(0), D(bi), P, acc);
        umma_tf(dim, D(1), D(br), P, true);
      }
    }
  } else {
    issue_step<GRAM>(s, st, 0, dre, dim, !first, bSameAsA);
    issue_step<GRAM>(s, st, 1, dre, dim, true, bSameAsA);
  }
}

// Commits of thread 0 that it has not yet seen arrive: at most one per stage
// barrier, since a stage is refilled (and committed again) only after its
// previous commit has been observed.
struct Pending {
  int c0 = -1, c1 = -1;   // chunk committed on bar[0] / bar[1], -1 when none is pending
  __device__ void committed(int ch) {
    if (ch & 1) c1 = ch;
    else c0 = ch;
  }
  __device__ void observed(int ch) {
    if (ch & 1) c1 = -1;
    else c0 = -1;
  }
  // After a timed-out wait: thread 0 waits, with the default poll count, for
  // every commit still pending, so that no MMA reads shared memory or writes
  // tensor memory after the kernel frees them and returns.
  __device__ void drain(USmem& s) const {
    if (c0 >= 0) mbar_wait(&s.bar[0], (unsigned)((c0 >> 1) & 1), kWaitPolls);
    if (c1 >= 0) mbar_wait(&s.bar[1], (unsigned)((c1 >> 1) & 1), kWaitPolls);
  }
};

// Main loop shared by both kernels: nch chunks; kofs(c, buf) fills s.kof[buf]
// for chunk c (threads < 32); load(c, buf) loads chunk c's operands into
// registers (A, and B unless bSameAsA); returns false when a wait timed out.
template <bool GRAM, bool TF, class KOfs, class Load>
__device__ __forceinline__ bool mainloop(USmem& s, int nch, Chunk& ca, Chunk& cb, bool conjA,
                                         bool conjB, bool bSameAsA, const KOfs& kofs,
                                         const Load& load, int polls) {
  const int tid = threadIdx.x;
  bool ok = true;
  Pending pend;
  if (nch > 0) load(0, 0);
  for (int c = 0; c < nch; ++c) {
    const int st = c & 1;
    if (c + 1 < nch) kofs(c + 1, (c + 1) & 1);
    if (c >= 2 && ok) {
      if (mbar_wait(&s.bar[st], (unsigned)(((c - 2) >> 1) & 1), polls)) pend.observed(c - 2);
      else ok = false;
    }
    if (ok) {
      store_operand<TF>(ca, &s.op[st][0][0], false, conjA);
      if (!bSameAsA) store_operand<TF>(cb, &s.op[st][0][0], true, conjB);
    }
    fence_async_smem();
    __syncthreads();
    if (c + 1 < nch) load(c + 1, (c + 1) & 1);
    if (tid == 0 && ok) {
      tc_fence_after();
      issue_chunk<GRAM, TF>(s, st, s.tmem, s.tmem + kTN, c == 0, bSameAsA);
      umma_commit(&s.bar[st]);
      pend.committed(c);
    }
    ok = __syncthreads_and(ok);
  }
  if (nch > 0 && ok) {
    const int l = nch - 1;
    if (mbar_wait(&s.bar[l & 1], (unsigned)((l >> 1) & 1), polls)) pend.observed(l);
    else ok = false;
  }
  ok = __syncthreads_and(ok);
  if (!ok && tid == 0) pend.drain(s);
  tc_fence_after();
  __syncthreads();
  return ok;
}

__device__ __forceinline__ void tmem_alloc(USmem& s) {
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     su32(&s.tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (threadIdx.x == 0) {
    mbar_init(&s.bar[0]);
    mbar_init(&s.bar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
}

__device__ __forceinline__ void tmem_free(USmem& s) {
  tc_fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(s.tmem),
                 "r"(kTmemCols)
                 : "memory");
}

// ---------------------------------------------------------------------------
template <bool TF>
__global__ void __launch_bounds__(kThr, 1)
    k_gram_umma(const cf* __restrict__ img, PatchMap m, cf* __restrict__ out, int nsplit,
                int lchunk, DevWait dw) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  USmem& s = *reinterpret_cast<USmem*>(smraw);
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
  const int a0 = ta * kTM, b0 = tb * kTN;
  const int l_begin = split * lchunk;
  const int l_end = min(m.L, l_begin + lchunk);
  const int n = m.n;
  const int nch = l_end > l_begin ? (l_end - l_begin + kKc - 1) / kKc : 0;
  tmem_alloc(s);
  for (int r = threadIdx.x; r < kTM; r += kThr) {
    const int a = a0 + r, b = b0 + r;
    s.rowA[r] = (a < n) ? (int)(m.tall ? (int64_t)a * ts : patch_off(m, a)) : -1;
    s.rowB[r] = (b < n) ? (int)(m.tall ? (int64_t)b * ts : patch_off(m, b)) : -1;
  }
  auto kofs = [&](int c, int buf) {
    if (threadIdx.x < kKc) {
      const int l = l_begin + c * kKc + threadIdx.x;
      s.kof[buf][threadIdx.x] = (l < l_end) ? (int)(m.tall ? patch_off(m, l) : (int64_t)l * ts) : -1;
    }
  };
  kofs(0, 0);
  __syncthreads();
  tc_fence_after();
  const cf* base = img + org;
  const bool cj = m.tall != 0;
  Chunk ca, cb;
  auto load = [&](int c, int buf) {
    (void)c;
    load_chunk(ca, base, s.rowA, s.kof[buf]);
    if (!diag) load_chunk(cb, base, s.rowB, s.kof[buf]);
  };
  const bool ok = mainloop<true, TF>(s, nch, ca, cb, cj, cj, diag, kofs, load, dw.polls);
  cf* G = out + ((nsplit > 1) ? (int64_t)split * n * n : ip * (int64_t)n * n);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a = a0 + (warp & 3) * 32 + lane;
  // on a time-out the tile is written as zeros (a zero Gram: the eigen stage
  // then finds no singular value above the threshold) and the error raised
  if (!ok && threadIdx.x == 0 && dw.err) atomicOr(dw.err, kErrMmaWait);
  {
    for (int cb = 0; cb < 4; ++cb) {
      const int col = (warp >> 2) * 64 + cb * 16;
      const uint32_t taddr = s.tmem + ((uint32_t)((warp & 3) * 32) << 16) + col;
      float re[16], im[16];
      if (ok && nch > 0) {
        tmem_ld16(taddr, re);
        tmem_ld16(taddr + kTN, im);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) re[j] = im[j] = 0.f;
      }
      if (a < n) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int b = b0 + col + j;
          if (b < n) {
            const cf v = make_float2(re[j], im[j]);
            G[(int64_t)b * n + a] = v;
            if (!diag) G[(int64_t)a * n + b] = cconj(v);
          }
        }
      }
    }
  }
  tmem_free(s);
}

// ---------------------------------------------------------------------------
template <bool TF>
__global__ void __launch_bounds__(kThr, 1)
    k_rebuild_umma(const cf* __restrict__ img, const cf* __restrict__ W, PatchMap m,
                   cf* __restrict__ out, int direct, DevWait dw) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  USmem& s = *reinterpret_cast<USmem*>(smraw);
  const int a0 = blockIdx.x * kTM, l0 = blockIdx.y * kTN;
  const int64_t ip = blockIdx.z;
  const int n = m.n;
  const cf* Wp = W + ip * (int64_t)n * n;
  const int64_t org = patch_origin(m, ip);
  const int64_t ts = tstride(m);
  const int nch = (n + kKc - 1) / kKc;
  tmem_alloc(s);
  // A rows a: the stored W column a holds conj(W[a][·]); conjugated back on conversion.
  // B rows l: M[·][l] — tall: conj(img[b·ts + org + off(l)]); wide: img[l·ts + org + off(b)]
  for (int r = threadIdx.x; r < kTM; r += kThr) {
    const int a = a0 + r, l = l0 + r;
    s.rowA[r] = (a < n) ? a * n : -1;
    s.rowB[r] = (l < m.L) ? (int)(m.tall ? patch_off(m, l) : (int64_t)l * ts) : -1;
  }
  // the K offsets of A (b) and B (frame or voxel of b) differ: A uses kof + its own rows
  auto kofs = [&](int c, int buf) {
    if (threadIdx.x < kKc) {
      const int b = c * kKc + threadIdx.x;
      s.kof[buf][threadIdx.x] = (b < n) ? (int)(m.tall ? (int64_t)b * ts : patch_off(m, b)) : -1;
    }
  };
  kofs(0, 0);
  __syncthreads();
  tc_fence_after();
  // A's element (a, b) is at Wp[a·n + b] (rows a·n in rowA, K offset b itself);
  // B's element (l, b) at org + rowB[l] + kof[b].
  Chunk ca, cb;
  auto load = [&](int c, int buf) {
#pragma unroll
    for (int i = 0; i < kPairs; ++i) {
      int r, k;
      pair_rk(i, r, k);
      const int ro = s.rowA[r];
#pragma unroll
      for (int d = 0; d < 2; ++d) {
        const int b = c * kKc + k + d;
        ca.v[i][d] = (ro >= 0 && b < n) ? __ldg(Wp + ro + b) : make_float2(0.f, 0.f);
      }
    }
    load_chunk(cb, img + org, s.rowB, s.kof[buf]);
  };
  const bool ok = mainloop<false, TF>(s, nch, ca, cb, true, m.tall != 0, false, kofs, load, dw.polls);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a = a0 + (warp & 3) * 32 + lane;
  // on a time-out the output tile is written as zeros and the error raised
  if (!ok && threadIdx.x == 0 && dw.err) atomicOr(dw.err, kErrMmaWait);
  {
    const int64_t offa = (a < n && !m.tall) ? patch_off(m, a) : 0;
    for (int cb = 0; cb < 4; ++cb) {
      const int col = (warp >> 2) * 64 + cb * 16;
      const uint32_t taddr = s.tmem + ((uint32_t)((warp & 3) * 32) << 16) + col;
      float re[16], im[16];
      if (ok && nch > 0) {
        tmem_ld16(taddr, re);
        tmem_ld16(taddr + kTN, im);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) re[j] = im[j] = 0.f;
      }
      if (a < n) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int l = l0 + col + j;
          if (l >= m.L) continue;
          if (m.tall) {   // frame a, voxel l: conj(M_out[a][l])
            const cf v = make_float2(re[j], -im[j]);
            if (direct) out[org + s.rowB[col + j] + (int64_t)a * ts] = v;
            else out[(ip * m.Nt + a) * (int64_t)m.p + l] = v;
          } else {        // frame l, voxel a
            const cf v = make_float2(re[j], im[j]);
            if (direct) out[org + offa + (int64_t)l * ts] = v;
            else out[(ip * m.Nt + l) * (int64_t)m.p + a] = v;
          }
        }
      }
    }
  }
  tmem_free(s);
}

}  // namespace

// The 32-bit row and K offset tables of the tcgen05 kernels cover this map.
bool umma_supported(const PatchMap& m) {
  const int64_t span = m.batch ? m.mstride : (int64_t)m.Nt * m.nvox;
  return span < (int64_t)0x7fffffff && (int64_t)m.n * m.n < (int64_t)0x7fffffff;
}

int umma_prepare() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  MSLR_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 64 && done[dev]) return MSLR_OK;
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_gram_umma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(USmem)));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_rebuild_umma<false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(USmem)));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_gram_umma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(USmem)));
  MSLR_CUDA_TRY(cudaFuncSetAttribute(k_rebuild_umma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(USmem)));
  if (dev < 64) done[dev] = true;
  return MSLR_OK;
}

int gram_umma_launch(const cf* img, const PatchMap& m, int64_t np, cf* out_or_part, int nsplit,
                     int lchunk, const DevWait& dw, cudaStream_t st, bool tf32) {
  if (int rc = umma_prepare()) return rc;
  const int T = (m.n + kTM - 1) / kTM;
  const int ntri = T * (T + 1) / 2;
  const dim3 grid(ntri, (unsigned)np, nsplit);
  if (tf32)
    k_gram_umma<true><<<grid, kThr, sizeof(USmem), st>>>(img, m, out_or_part, nsplit, lchunk, dw);
  else
    k_gram_umma<false><<<grid, kThr, sizeof(USmem), st>>>(img, m, out_or_part, nsplit, lchunk, dw);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int rebuild_umma_launch(const cf* img, const cf* W, const PatchMap& m, int64_t np, cf* out,
                        int direct, const DevWait& dw, cudaStream_t st, bool tf32) {
  if (int rc = umma_prepare()) return rc;
  const dim3 grid((m.n + kTM - 1) / kTM, (m.L + kTN - 1) / kTN, (unsigned)np);
  if (tf32)
    k_rebuild_umma<true><<<grid, kThr, sizeof(USmem), st>>>(img, W, m, out, direct, dw);
  else
    k_rebuild_umma<false><<<grid, kThr, sizeof(USmem), st>>>(img, W, m, out, direct, dw);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

}  // namespace mslr
