// setup.cu — the data set-up of run_recon on the device (sm_100a).
//
// scripts/reconstruct.jl:86-147 prepares the inputs of the iteration on the
// host: coil maps normalised to unit sum of squares (:89), the k-space scaled
// by the 99th percentile of |sense_comb| (:100-104, src/recon.jl:310-321),
// the sampling mask taken from coil 1 and checked against every coil and
// frame (:109-118), and the sampled values gathered into (K, Nc, Nt) (:144-147).
// Here each step is a kernel:
//   k_sos_norm     S ./ (sqrt(Σ_c |S_c|²) + eps(Float32)), Float32, coils in order
//   k_mask_count   per (frame, chunk of voxels): Ω from coil 1, every coil's
//                  nonzero pattern compared with it, samples counted
//   k_compact      idx (0-based, ascending) and y = ksp[idx] per frame, from
//                  the per-chunk offsets (exclusive scan on the host)
//   k_comb_abs     |A'y / √Nvox / (Σ_c |S_c|² + eps())| as Float32 — the
//                  magnitude of sense_comb, whose ifft part equals the exact
//                  adjoint of the centred forward DFT divided by Nvox
//   k_radix_hist   11-bit histograms of the magnitudes' bit patterns under a
//                  prefix: three passes give an exact order statistic
//   k_scale        y = Float32(Float64(y) / max(q, eps(Float32)))
// Counts and offsets are integers, so idx and y are bit-exact; the
// percentile is the exact type-7 quantile of the magnitudes computed here.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace mslr {

namespace {

constexpr int kChunk = 1024;   // voxels per block in the mask kernels

__global__ void k_sos_norm(const cf* __restrict__ in, cf* __restrict__ out, int Nc, int64_t nvox) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvox;
       v += (int64_t)gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int c = 0; c < Nc; ++c) {
      const cf s = in[c * nvox + v];
      acc = acc + __fadd_rn(__fmul_rn(s.x, s.x), __fmul_rn(s.y, s.y));
    }
    const float den = __fadd_rn(__fsqrt_rn(acc), 1.1920928955078125e-7f);
    for (int c = 0; c < Nc; ++c) {
      const cf s = in[c * nvox + v];
      out[c * nvox + v] = make_float2(__fdiv_rn(s.x, den), __fdiv_rn(s.y, den));
    }
  }
}

__device__ __forceinline__ bool nz(cf v) { return v.x != 0.f || v.y != 0.f; }

// grid (chunks, Nt), kChunk threads.  cnt[t·chunks + b] = samples in the chunk;
// *bad_coil = smallest coil index whose pattern differs (atomicMin).
__global__ void __launch_bounds__(kChunk) k_mask_count(const cf* __restrict__ ksp, int Nc, int64_t nvox,
                                                       int* __restrict__ cnt, int* __restrict__ bad_coil) {
  __shared__ int wsum[kChunk / 32];
  const int t = blockIdx.y;
  const int64_t v = (int64_t)blockIdx.x * kChunk + threadIdx.x;
  bool m = false;
  if (v < nvox) {
    const cf* base = ksp + (int64_t)t * Nc * nvox + v;
    m = nz(base[0]);
    for (int c = 1; c < Nc; ++c)
      if (nz(base[c * nvox]) != m) {
        atomicMin(bad_coil, c);
        break;
      }
  }
  const unsigned b = __ballot_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = __popc(b);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < kChunk / 32; ++w) s += wsum[w];
    cnt[t * gridDim.x + blockIdx.x] = s;
  }
}

// grid (chunks, Nt): idx[t][off + rank] = v, y[t][c][off + rank] = ksp[t][c][v]
__global__ void __launch_bounds__(kChunk) k_compact(const cf* __restrict__ ksp, int Nc, int64_t nvox,
                                                    const int64_t* __restrict__ off, int64_t K,
                                                    int32_t* __restrict__ idx, cf* __restrict__ y) {
  __shared__ int wsum[kChunk / 32];
  const int t = blockIdx.y;
  const int64_t v = (int64_t)blockIdx.x * kChunk + threadIdx.x;
  const cf* base = ksp + (int64_t)t * Nc * nvox;
  const bool m = (v < nvox) && nz(base[v]);
  const unsigned b = __ballot_sync(0xffffffffu, m);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wsum[w] = __popc(b);
  __syncthreads();
  int before = 0;
  for (int q = 0; q < w; ++q) before += wsum[q];
  if (!m) return;
  const int64_t k = off[t * gridDim.x + blockIdx.x] + before + __popc(b & ((1u << lane) - 1u));
  if (k >= K) return;
  idx[(int64_t)t * K + k] = (int32_t)v;
  for (int c = 0; c < Nc; ++c) y[((int64_t)t * Nc + c) * K + k] = base[c * nvox + v];
}

// mag[t][v] = |ahy[t][v] · s / (Σ_c |S_c(v)|² + eps())|, Float64 then Float32
__global__ void k_comb_abs(const cf* __restrict__ ahy, const cf* __restrict__ smaps, int Nc, int64_t nvox,
                           int64_t total, double s, float* __restrict__ mag) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = q % nvox;
    float den32 = 0.f;
    for (int c = 0; c < Nc; ++c) {
      const cf a = smaps[c * nvox + v];
      den32 = __fadd_rn(den32, __fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)));
    }
    const double den = (double)den32 + 2.220446049250313e-16;
    const cf n = ahy[q];
    const float re = (float)((double)n.x * s / den), im = (float)((double)n.y * s / den);
    mag[q] = (float)sqrt((double)re * re + (double)im * im);
  }
}

// hist[d] += #{ i : (bits_i >> shift) mod 2^width == d  and  bits_i >> (shift + width) == prefix }
__global__ void k_radix_hist(const float* __restrict__ mag, int64_t n, int shift, int width,
                             uint32_t prefix, unsigned long long* __restrict__ hist) {
  __shared__ unsigned int h[2048];
  for (int i = threadIdx.x; i < 2048; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const int hs = shift + width;
  const uint32_t mask = (1u << width) - 1u;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t b = __float_as_uint(mag[i]);
    if (hs >= 32 || (b >> hs) == prefix) atomicAdd(&h[(b >> shift) & mask], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 2048; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

__global__ void k_scale(cf* __restrict__ y, int64_t n, double div, int* __restrict__ underflow) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const cf v = y[i];
    const cf o = make_float2((float)((double)v.x / div), (float)((double)v.y / div));
    if (nz(v) && !nz(o)) atomicOr(underflow, 1);
    y[i] = o;
  }
}

// the element of rank j (0-based, ascending) among the n non-negative floats
int order_stat(const float* mag, int64_t n, int64_t j, unsigned long long* hist, float* out,
               cudaStream_t st) {
  uint32_t prefix = 0;
  int64_t rank = j;
  std::vector<unsigned long long> h(2048);
  const int shifts[3] = {21, 10, 0};
  const int widths[3] = {11, 11, 10};
  for (int p = 0; p < 3; ++p) {
    MSLR_CUDA_TRY(cudaMemsetAsync(hist, 0, 2048 * sizeof(unsigned long long), st));
    k_radix_hist<<<1184, 256, 0, st>>>(mag, n, shifts[p], widths[p], prefix, hist);
    MSLR_CUDA_TRY(cudaGetLastError());
    MSLR_CUDA_TRY(cudaMemcpyAsync(h.data(), hist, 2048 * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, st));
    MSLR_CUDA_TRY(cudaStreamSynchronize(st));
    int d = 0;
    const int nb = 1 << widths[p];
    for (; d < nb; ++d) {
      if (rank < (int64_t)h[d]) break;
      rank -= (int64_t)h[d];
    }
    if (d == nb) return fail(MSLR_ERR_CUDA, "order statistic out of range");
    prefix = (prefix << widths[p]) | (uint32_t)d;
  }
  uint32_t bits = prefix;
  std::memcpy(out, &bits, sizeof(float));
  return MSLR_OK;
}

}  // namespace

int sos_normalize(const int N[3], int Nc, const cf* in, cf* out, cudaStream_t st) {
  const int64_t nvox = (int64_t)N[0] * N[1] * N[2];
  k_sos_norm<<<1184, 256, 0, st>>>(in, out, Nc, nvox);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

// Ω from coil 1 and the reference's two checks; K = samples per frame.  With
// idx / y given (capacity K_cap per frame) the samples are also gathered.
int sampling(const int N[3], int Nc, int Nt, const cf* ksp, int64_t* K, int32_t* idx, cf* y,
             int64_t K_cap, cudaStream_t st) {
  const int64_t nvox = (int64_t)N[0] * N[1] * N[2];
  const int chunks = (int)((nvox + kChunk - 1) / kChunk);
  const size_t ncnt = (size_t)chunks * Nt;
  int* d_cnt = nullptr;
  int64_t* d_off = nullptr;
  MSLR_CUDA_TRY(cudaMallocAsync((void**)&d_cnt, ncnt * sizeof(int) + sizeof(int), st));
  int* d_bad = d_cnt + ncnt;
  std::vector<int> h(ncnt);
  int bad = 0;
  int rc = MSLR_OK;
  const int big = 1 << 30;
  cudaError_t e = cudaMemcpyAsync(d_bad, &big, sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    k_mask_count<<<dim3(chunks, Nt), kChunk, 0, st>>>(ksp, Nc, nvox, d_cnt, d_bad);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d_cnt, ncnt * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) rc = fail(MSLR_ERR_CUDA, cudaGetErrorString(e));
  std::vector<int64_t> off(ncnt);
  int64_t k0 = -1;
  if (!rc && bad != big)   // scripts/reconstruct.jl:113-115 (1-based coil number)
    rc = fail(MSLR_ERR_ARG, "Coil " + std::to_string(bad + 1) + " has a different sampling pattern");
  for (int t = 0; !rc && t < Nt; ++t) {
    int64_t s = 0;
    for (int b = 0; b < chunks; ++b) {
      off[(size_t)t * chunks + b] = s;
      s += h[(size_t)t * chunks + b];
    }
    if (t > 0 && s != k0)   // :116-118
      rc = fail(MSLR_ERR_ARG, "Frame " + std::to_string(t + 1) + " has a different sample count");
    k0 = s;
  }
  if (!rc) *K = k0;
  if (!rc && (idx || y)) {
    if (!idx || !y) rc = fail(MSLR_ERR_ARG, "idx and y must both be given");
    else if (k0 > K_cap) rc = fail(MSLR_ERR_ARG, "sample capacity too small: need " + std::to_string(k0));
  }
  if (!rc && idx) {
    e = cudaMallocAsync((void**)&d_off, ncnt * sizeof(int64_t), st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_off, off.data(), ncnt * sizeof(int64_t), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
      k_compact<<<dim3(chunks, Nt), kChunk, 0, st>>>(ksp, Nc, nvox, d_off, k0, idx, y);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fail(MSLR_ERR_CUDA, cudaGetErrorString(e));
  }
  if (d_off) cudaFreeAsync(d_off, st);
  cudaFreeAsync(d_cnt, st);
  cudaStreamSynchronize(st);
  return rc;
}

// After mslr_bind with the unscaled samples: scale factor = quantile(|sense_comb|, 0.99)
// (type 7), y ← y / max(q, eps(Float32)) in place, and the context rebound.
int prepare_scale(Ctx* c, const cf* smaps, cf* y, const int32_t* idx, double* scale_out, cudaStream_t st) {
  const int64_t total = (int64_t)c->Nt * c->nvox;
  float* mag = reinterpret_cast<float*>(c->d_img_tmp);   // Nt·Nvox floats fit an image of c64
  unsigned long long* hist = nullptr;
  int* d_uf = nullptr;
  MSLR_CUDA_TRY(cudaMallocAsync((void**)&hist, 2048 * sizeof(unsigned long long) + 16, st));
  d_uf = reinterpret_cast<int*>(hist + 2048);
  int rc = MSLR_OK;
  k_comb_abs<<<1184, 256, 0, st>>>(c->d_ahy, smaps, c->Nc, c->nvox, total,
                                   1.0 / std::sqrt((double)c->nvox), mag);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) rc = fail(MSLR_ERR_CUDA, cudaGetErrorString(e));
  // Statistics.quantile, type 7: h = (n − 1)p, a = v[⌊h⌋], b = v[⌊h⌋ + 1]
  const double h = (double)(total - 1) * 0.99;
  const int64_t j = (int64_t)std::floor(h);
  const double g = h - (double)j;
  float a = 0.f, b = 0.f;
  if (!rc) rc = order_stat(mag, total, j, hist, &a, st);
  if (!rc) rc = (j + 1 < total) ? order_stat(mag, total, j + 1, hist, &b, st) : (b = a, MSLR_OK);
  double q = 0.0;
  if (!rc) {
    const float d = b - a;
    q = (double)a + g * (double)d;
    *scale_out = q;
    const double div = std::max(q, (double)1.1920928955078125e-7);
    int uf = 0;
    e = cudaMemsetAsync(d_uf, 0, sizeof(int), st);
    if (e == cudaSuccess) {
      k_scale<<<1184, 256, 0, st>>>(y, (int64_t)c->Nt * c->Nc * c->K, div, d_uf);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&uf, d_uf, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fail(MSLR_ERR_CUDA, cudaGetErrorString(e));
    else if (uf)
      rc = fail(MSLR_ERR_ARG, "a k-space sample underflows to zero under the scale factor");
  }
  cudaFreeAsync(hist, st);
  cudaStreamSynchronize(st);
  if (!rc) rc = sense_bind(c, smaps, y, idx, 0, st);
  return rc;
}

}  // namespace mslr
