// common.cuh — shared types and helpers of libmslr (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/mslr.h"

namespace mslr {

typedef float2 cf;    // ComplexF32, interleaved (re, im)
typedef double2 cd;   // ComplexF64

__host__ __device__ __forceinline__ cf cmk(float r, float i) { return make_float2(r, i); }
__host__ __device__ __forceinline__ cf cadd(cf a, cf b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cf csub(cf a, cf b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cf cmul(cf a, cf b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__host__ __device__ __forceinline__ cf cmulc(cf a, cf b) {
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ cf cconj(cf a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ cf cscale(cf a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float cabs2(cf a) { return a.x * a.x + a.y * a.y; }

__host__ __device__ __forceinline__ cd dmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ cd dadd(cd a, cd b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cd dsub(cd a, cd b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cd dmul(cd a, cd b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cd dconj(cd a) { return make_double2(a.x, -a.y); }

// Maximum FFT axis length handled by the shared-memory FFT.
constexpr int kMaxFftLen = 1024;
constexpr int kMaxPasses = 12;

// Mixed-radix plan of one axis (Stockham passes).
struct AxisPlan {
  int n;
  int npass;
  int radix[kMaxPasses];
};

// Geometry of one patch scale (src/recon.jl:54-72), all 0-based.
struct ScaleGeom {
  int ps[3];        // clamped patch size
  int ss[3];        // stride
  int nsteps[3];    // cld(N - ps, ss)
  int64_t Np;       // number of patches
  int p;            // prod(ps)
  int n;            // min(p, Nt): side of the Gram matrix
  int L;            // max(p, Nt): contraction length of the Gram
  bool tall;        // p >= Nt: Gram = P^H P (time x time); else P P^H (voxel x voxel)
  bool partition;   // patches tile the volume exactly (no overlap, no gaps)
  bool global;      // one patch covering the whole volume
  int* d_starts;    // device: x-starts, y-starts, z-starts (nsteps+1 each)
  // coverage ranges per dim for the gather recombine: for coordinate c in dim d,
  // covering patch indices along d are [lo, hi] (inclusive); -1 if none
  int* d_cover;     // device: per dim, 2*N[d] ints
  int nsplit_tuned = 0;   // split-K count of the Gram chosen by the autotuner (0: heuristic)
  int eig_big = 0;        // eigen stage in the 1024-thread CTA variant (autotuner; n > 384 always is)
  std::vector<int> h_starts;
};

// Status helpers -------------------------------------------------------------
struct Status {
  int code = MSLR_OK;
  std::string msg;
};

// Bits of a device error word (one int32 per context, or per call of the
// context-free batched SVST).  Kernels set them with atomicOr; the host reads
// and clears the word when a call synchronises.
constexpr int kErrIdxRange = 1;    // bind: a sample index outside the grid
constexpr int kErrIdxOrder = 2;    // bind: indices not strictly ascending
constexpr int kErrNonfinite = 4;   // NaN / Inf in the POGM restart sums
constexpr int kErrBulkWait = 8;    // a SENSE kernel's wait for a bulk copy timed out
constexpr int kErrMmaWait = 16;    // a tcgen05 kernel's wait for its MMAs timed out

// Default poll count of a bounded mbarrier wait (a few tens of ms on B200).
constexpr int kWaitPolls = 1 << 22;

// Where a kernel with bounded waits reports a time-out, and how many polls a
// wait makes before it gives up.  `polls` is settable (mslr_set_wait_limit)
// so that a test can make a wait run out; the wait that drains in-flight
// work before a kernel returns always uses kWaitPolls.
struct DevWait {
  int* err = nullptr;
  int polls = kWaitPolls;
};

}  // namespace mslr

#define MSLR_CUDA_TRY(expr)                                                        \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      return ::mslr::fail(MSLR_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    }                                                                              \
  } while (0)
