// umma.cuh — building blocks of the tcgen05 (5th-generation tensor core)
// kernels: shared-memory matrix descriptors, instruction descriptors, MMA
// issue and commit, tensor-memory allocation and loads, mbarriers with
// bounded waits, and the split of FP32 values into BF16 hi / lo parts.
//
// Operand tiles use the unswizzled ("interleave") canonical layouts of
// 8 × 8-element core matrices of 128 bytes:
//   K-major  element (r, k) at ((r / 8)·KC + k / 8)·64 + (r % 8)·8 + k % 8
//   MN-major element (r, k) at ((r / 8)·KC + k / 8)·64 + (k % 8)·8 + r % 8
// (bf16 units, KC = K / 8 cores per 8-row group): the leading byte offset
// (next core along K) is 128 bytes and the stride byte offset (next group of
// 8 rows along M or N) is KC·128 bytes in both.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace mslr {
namespace umma {

__device__ __forceinline__ unsigned su32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor (sm_100 layout, version 1, no swizzle)
__device__ __forceinline__ uint64_t sdesc(const void* p, unsigned lbo, unsigned sbo) {
  const uint64_t a = su32(p);
  return ((a >> 4) & 0x3FFFull) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: BF16 × BF16 → F32, M × N, optional
// negation of A / B and MN-major A / B
__host__ __device__ constexpr uint32_t idesc(int M, int N, bool negA, bool negB, bool aMN, bool bMN) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((negA ? 1u : 0u) << 13) | ((negB ? 1u : 0u) << 14) |
         ((aMN ? 1u : 0u) << 15) | ((bMN ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t id, bool acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(a), "l"(b), "r"(id), "r"(acc ? 1u : 0u));
}
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   su32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(su32(bar)) : "memory");
}
// bounded wait for the phase of `bar` with the given parity; false on time-out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const unsigned a = su32(bar);
  for (int it = 0; it < (1 << 22); ++it) {
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
// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32·(w % 4)..)
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
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
// warp 0 allocates `cols` TMEM columns (a power of two >= 32); address into *dst
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, unsigned cols) {
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     su32(dst)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
}
// all threads: finish TMEM use; warp 0 frees the columns
__device__ __forceinline__ void tmem_free(uint32_t taddr, unsigned cols) {
  fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(cols)
                 : "memory");
}

// hi / lo split of two values into packed bf16 pairs (first value in the low half)
__device__ __forceinline__ void split_pair(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

}  // namespace umma
}  // namespace mslr
