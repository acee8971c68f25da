// probe.cu — measured FP32 FMA throughput of the device, the denominator of
// the SIMT-bound kernels' roofline fractions (the SENSE FFT passes and the
// eigen stage).  No counterpart in the reference.
#include <algorithm>

#include "internal.h"

namespace mslr {
namespace {

constexpr int kChains = 8;     // independent FMA chains per thread
constexpr int kIters = 4096;   // dependent FMAs per chain

// Every thread runs kChains independent chains of kIters dependent FMAs; the
// result is stored (when it cannot be zero) so that the chains are not removed.
__global__ void __launch_bounds__(256) k_fma(float* out, float a, float b) {
  float v[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) v[c] = (float)(threadIdx.x + c);
#pragma unroll 16
  for (int i = 0; i < kIters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = fmaf(v[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += v[c];
  if (s == 1234.5678f) out[blockIdx.x] = s;
}

}  // namespace

int fp32_peak_probe(double* tflops, cudaStream_t st) {
  int dev = 0, nsm = 0;
  MSLR_CUDA_TRY(cudaGetDevice(&dev));
  MSLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = nsm * 8;   // 8 CTAs of 256 threads per SM: 64 warps resident
  float* out = nullptr;
  MSLR_CUDA_TRY(cudaMalloc(&out, blocks * sizeof(float)));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  double best = 0.0;
  if (e == cudaSuccess) {
    k_fma<<<blocks, 256, 0, st>>>(out, 0.999f, 0.001f);   // warm-up
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
      cudaEventRecord(e0, st);
      k_fma<<<blocks, 256, 0, st>>>(out, 0.999f, 0.001f);
      cudaEventRecord(e1, st);
      e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e == cudaSuccess && ms > 0.f) {
        const double flops = 2.0 * kChains * kIters * 256.0 * blocks;
        best = std::max(best, flops / (ms * 1e-3) / 1e12);
      }
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess) return fail(MSLR_ERR_CUDA, std::string("FP32 peak probe: ") + cudaGetErrorString(e));
  *tflops = best;
  return MSLR_OK;
}

}  // namespace mslr

extern "C" int mslr_fp32_peak(double* tflops, void* stream) {
  if (!tflops) return mslr::fail(MSLR_ERR_ARG, "null output pointer");
  return mslr::fp32_peak_probe(tflops, reinterpret_cast<cudaStream_t>(stream));
}
