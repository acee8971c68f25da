// cost.cu — data-consistency cost of run_recon (scripts/reconstruct.jl:176-178)
// without keeping the raw k-space on the device.
//
//   dc_cost(X) = ½ ‖A x̄ − y‖²,  x̄ = Σ_k X_k
//              = ½ (Re⟨x̄, g⟩ − Re⟨x̄, A'y⟩ + ‖y‖²),   g = A'A x̄ − A'y,
// because ‖A x̄‖² = ⟨x̄, A'A x̄⟩ = ⟨x̄, g⟩ + ⟨x̄, A'y⟩.  g comes from one normal
// operator, A'y and ‖y‖² are kept from bind.  All sums are FP64: per-thread,
// per-block in a fixed order, then over blocks on the host in block order.
#include <vector>

#include "internal.h"

namespace mslr {

namespace {

constexpr int kBlocks = 592;   // 4 per SM
constexpr int kThreads = 256;

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block sum in warp order; thread 0 holds the result
__device__ __forceinline__ double block_sum_d(double v, double* red) {
  v = warp_sum_d(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  __syncthreads();
  return s;
}

__global__ void __launch_bounds__(kThreads) k_sumsq(const cf* __restrict__ y, int64_t n,
                                                    double* __restrict__ part) {
  __shared__ double red[kThreads / 32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const cf v = y[i];
    s += (double)v.x * v.x + (double)v.y * v.y;
  }
  s = block_sum_d(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Re⟨x̄, g⟩ and Re⟨x̄, a⟩ with x̄ = Σ_k X_k summed in FP32 as the reference's sum(X)
__global__ void __launch_bounds__(kThreads) k_cost_dots(const cf* __restrict__ X, int ns,
                                                        int64_t sstride, const cf* __restrict__ g,
                                                        const cf* __restrict__ a, int64_t E,
                                                        double* __restrict__ part) {
  __shared__ double red[kThreads / 32];
  double s1 = 0.0, s2 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < E;
       i += (int64_t)gridDim.x * blockDim.x) {
    cf x = X[i];
    for (int k = 1; k < ns; ++k) x = cadd(x, X[i + k * sstride]);
    const cf gv = g[i], av = a[i];
    s1 += (double)x.x * gv.x + (double)x.y * gv.y;
    s2 += (double)x.x * av.x + (double)x.y * av.y;
  }
  s1 = block_sum_d(s1, red);
  s2 = block_sum_d(s2, red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1;
    part[2 * blockIdx.x + 1] = s2;
  }
}

int ensure_part(Ctx* c) {
  if (c->d_cost_part) return MSLR_OK;
  return dalloc(c, (void**)&c->d_cost_part, 2 * kBlocks * sizeof(double));
}

}  // namespace

// ‖y‖² of a (K, Nc, Nt) k-space array, FP64.  Synchronises st.
int data_norm2(Ctx* c, const cf* y, double* out, cudaStream_t st) {
  int rc;
  if ((rc = ensure_part(c))) return rc;
  const int64_t n = (int64_t)c->K * c->Nc * c->Nt;
  k_sumsq<<<kBlocks, kThreads, 0, st>>>(y, n, c->d_cost_part);
  MSLR_CUDA_TRY(cudaGetLastError());
  c->launches += 1;
  std::vector<double> h(kBlocks);
  MSLR_CUDA_TRY(cudaMemcpyAsync(h.data(), c->d_cost_part, kBlocks * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  double s = 0.0;
  for (double v : h) s += v;
  *out = s;
  return MSLR_OK;
}

// dc_cost(X) for X (ns, Nt, Nz, Ny, Nx).  Synchronises st.
int dc_cost_eval(Ctx* c, const cf* X, int ns, double* dc_out, cudaStream_t st) {
  int rc;
  const int64_t E = (int64_t)c->Nt * c->nvox;
  if (!c->d_cost_g && (rc = dalloc(c, (void**)&c->d_cost_g, (size_t)E * sizeof(cf)))) return rc;
  if ((rc = ensure_part(c))) return rc;
  // the cost is a difference of terms ~‖y‖² that cancel as the iterate
  // converges: evaluate it with the FP32 FFT plane pass, not the split-BF16
  // tensor-core one
  const bool tc = c->xy_tc;
  c->xy_tc = false;
  rc = normal_op(c, X, ns, E, c->d_cost_g, true, st);
  c->xy_tc = tc;
  if (rc) return rc;
  k_cost_dots<<<kBlocks, kThreads, 0, st>>>(X, ns, E, c->d_cost_g, c->d_ahy, E, c->d_cost_part);
  MSLR_CUDA_TRY(cudaGetLastError());
  c->launches += 1;
  std::vector<double> h(2 * kBlocks);
  MSLR_CUDA_TRY(cudaMemcpyAsync(h.data(), c->d_cost_part, 2 * kBlocks * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  double s1 = 0.0, s2 = 0.0;
  for (int b = 0; b < kBlocks; ++b) {
    s1 += h[2 * b];
    s2 += h[2 * b + 1];
  }
  *dc_out = 0.5 * (s1 - s2 + c->ynorm2);
  return MSLR_OK;
}

}  // namespace mslr
