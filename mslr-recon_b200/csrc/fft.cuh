// fft.cuh — shared-memory mixed-radix Stockham FFT over batches of lines.
//
// The SENSE operator's centred 3-D DFT (src/sense_gpu.jl:75, :93) is done as
// three 1-D passes whose lines are staged in shared memory.  A line of length
// n = R_0 R_1 ... R_{P-1} is transformed by P Stockham passes (autosort, no
// digit reversal), ping-ponging between two shared buffers of identical
// layout: element e of line l lives at  l*ls + e*es.
//
// Forward uses w = exp(-2πi/n); inverse is the unnormalised backward
// transform (exp(+2πi/n)).  Twiddles come from a per-axis table
// tw[k] = exp(-2πi k/n) computed on the host in double precision.
#pragma once
#include "common.cuh"

namespace mslr {

template <bool INV>
__device__ __forceinline__ cf tw_get(const cf* tw, int k) {
  cf w = tw[k];
  return INV ? cconj(w) : w;
}

// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ cf rot_mi(cf a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ void dft2(cf* v) {
  cf a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <bool INV>
__device__ __forceinline__ void dft3(cf* v) {
  const float s3 = 0.86602540378443864676f;  // sin(2π/3)
  cf a = v[0], b = v[1], c = v[2];
  cf t = cadd(b, c);
  cf m = make_float2(a.x - 0.5f * t.x, a.y - 0.5f * t.y);
  cf d = cscale(csub(b, c), s3);
  cf id = rot_mi<INV>(d);  // ∓i·(√3/2)(b − c)
  v[0] = cadd(a, t);
  v[1] = cadd(m, id);
  v[2] = csub(m, id);
}

template <bool INV>
__device__ __forceinline__ void dft4(cf* v) {
  cf a = v[0], b = v[1], c = v[2], d = v[3];
  cf s0 = cadd(a, c), d0 = csub(a, c);
  cf s1 = cadd(b, d), d1 = rot_mi<INV>(csub(b, d));
  v[0] = cadd(s0, s1);
  v[1] = cadd(d0, d1);
  v[2] = csub(s0, s1);
  v[3] = csub(d0, d1);
}

template <bool INV>
__device__ __forceinline__ void dft5(cf* v) {
  const float c1 = 0.30901699437494742410f;   // cos(2π/5)
  const float c2 = -0.80901699437494742410f;  // cos(4π/5)
  const float s1 = 0.95105651629515357212f;   // sin(2π/5)
  const float s2 = 0.58778525229247312917f;   // sin(4π/5)
  cf x0 = v[0];
  cf t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
  cf t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
  cf a1 = make_float2(x0.x + c1 * t1.x + c2 * t2.x, x0.y + c1 * t1.y + c2 * t2.y);
  cf a2 = make_float2(x0.x + c2 * t1.x + c1 * t2.x, x0.y + c2 * t1.y + c1 * t2.y);
  cf b1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
  cf b2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
  cf ib1 = rot_mi<INV>(b1), ib2 = rot_mi<INV>(b2);
  v[0] = cadd(x0, cadd(t1, t2));
  v[1] = cadd(a1, ib1);
  v[4] = csub(a1, ib1);
  v[2] = cadd(a2, ib2);
  v[3] = csub(a2, ib2);
}

constexpr int kMaxRadix = 16;

// Generic small-prime DFT through the axis twiddle table (n divisible by R).
template <bool INV>
__device__ __forceinline__ void dft_generic(cf* v, int R, const cf* tw, int n) {
  cf out[kMaxRadix];
  const int step = n / R;
  for (int q = 0; q < R; ++q) {
    cf acc = v[0];
    for (int r = 1; r < R; ++r) {
      cf w = tw_get<INV>(tw, ((r * q) % R) * step);
      acc = cadd(acc, cmul(v[r], w));
    }
    out[q] = acc;
  }
  for (int q = 0; q < R; ++q) v[q] = out[q];
}

// One Stockham pass over all lines.  src/dst use the same (es, ls) layout.
template <bool INV>
__device__ __forceinline__ void stockham_pass(const cf* __restrict__ src, cf* __restrict__ dst,
                                              int n, int R, int Ns, const cf* tw, int nlines,
                                              int es, int ls) {
  const int m = n / R;
  const int total = nlines * m;
  const int twstep = n / (Ns * R);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int line = idx / m;
    const int j = idx - line * m;
    const int k = j % Ns;
    const cf* s = src + (size_t)line * ls;
    cf v[kMaxRadix];
#pragma unroll 4
    for (int r = 0; r < R; ++r) v[r] = s[(j + r * m) * es];
    if (Ns > 1) {
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw_get<INV>(tw, (r * k * twstep) % n));
    }
    switch (R) {
      case 2: dft2<INV>(v); break;
      case 3: dft3<INV>(v); break;
      case 4: dft4<INV>(v); break;
      case 5: dft5<INV>(v); break;
      default: dft_generic<INV>(v, R, tw, n); break;
    }
    const int base = (j / Ns) * Ns * R + k;
    cf* d = dst + (size_t)line * ls;
#pragma unroll 4
    for (int r = 0; r < R; ++r) d[(base + r * Ns) * es] = v[r];
  }
}

// Transform `nlines` lines held in buffer a (scratch b of the same layout).
// Returns the buffer holding the result (a or b).  Ends with __syncthreads().
template <bool INV>
__device__ cf* fft_lines(cf* a, cf* b, const AxisPlan& pl, const cf* tw, int nlines, int es, int ls) {
  cf* src = a;
  cf* dst = b;
  int Ns = 1;
  for (int p = 0; p < pl.npass; ++p) {
    const int R = pl.radix[p];
    stockham_pass<INV>(src, dst, pl.n, R, Ns, tw, nlines, es, ls);
    __syncthreads();
    Ns *= R;
    cf* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

}  // namespace mslr
