// fft_fast.cuh — register-resident mixed-radix FFT passes for the tuned form.
//
// A line of length n = R_0 · R_1 (· R_2) is transformed by Stockham passes in
// which each thread owns exactly one radix-R butterfly: it loads its R inputs
// (from shared memory or straight from global memory), applies twiddles, does
// the R-point DFT in registers and stores its R outputs.  Passes alternate
// between two shared buffers, so one barrier per pass suffices.  Radices up
// to 12 are built at compile time from 2, 3, 4 and 5; the reference's image
// axes (90, 60, 48, 32, 24 ...) take two passes each.
//
// Index convention (Stockham autosort, natural order in and out): pass with
// radix R after radices of product Ns, thread j < m = n/R, k = j mod Ns:
//   in  : x[j + r·m] · w^{r·k·n/(Ns·R)},  r < R
//   out : y[(j/Ns)·Ns·R + k + r·Ns] = DFT_R(in)[r]
// All index divisions are by per-pass constants and use exact multiply-shift
// reciprocals (valid for dividends and divisors below 1024).
#pragma once
#include "fft.cuh"

namespace mslr {
namespace fast {

constexpr int kMaxThreads = 1024;

// (x · M) >> 21 == x / d for 0 <= x < 1024, 1 <= d <= 1024, M = 2^21/d + 1
__host__ __device__ constexpr unsigned recip(int d) { return (1u << 21) / (unsigned)d + 1u; }
__device__ __forceinline__ int fdiv(int x, unsigned M) { return (int)(((unsigned)x * M) >> 21); }

// Host-computed description of one pass.
struct FPass {
  int R;         // radix
  int m;         // n / R: butterflies per line
  int Ns;        // product of the radices of the earlier passes
  int twstep;    // n / (Ns·R)
  unsigned Mm;   // recip(m)
  unsigned Mns;  // recip(Ns)
};

// A 1-D transform of `nlines` lines of length n: forward passes in order and
// inverse passes in reversed radix order (so that the last forward pass and
// the first inverse pass share a radix and can be fused around a mask).
struct FPlan {
  int n, npass, nlines;
  unsigned Mnl;   // recip(nlines)
  FPass fw[3];
  FPass iv[3];
};

// ---- R-point DFTs in registers ---------------------------------------------
// `step` = n/R, the stride of ω_R in the axis twiddle table tw[k] = e^{-2πik/n}.
template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<2, INV> {
  static __device__ __forceinline__ void run(cf* v, const cf*, int) { dft2<INV>(v); }
};
template <bool INV>
struct Dft<3, INV> {
  static __device__ __forceinline__ void run(cf* v, const cf*, int) { dft3<INV>(v); }
};
template <bool INV>
struct Dft<4, INV> {
  static __device__ __forceinline__ void run(cf* v, const cf*, int) { dft4<INV>(v); }
};
template <bool INV>
struct Dft<5, INV> {
  static __device__ __forceinline__ void run(cf* v, const cf*, int) { dft5<INV>(v); }
};

// R = A·B in registers: r = r1 + A·r2, q = q2 + B·q1,
// X[q] = Σ_{r1} ω_A^{r1 q1} · ω_R^{r1 q2} · Σ_{r2} x[r1 + A r2] ω_B^{r2 q2}.
template <int A, int B, bool INV>
struct DftCT {
  static __device__ __forceinline__ void run(cf* v, const cf* tw, int step) {
    cf t[A][B];
#pragma unroll
    for (int r1 = 0; r1 < A; ++r1) {
#pragma unroll
      for (int r2 = 0; r2 < B; ++r2) t[r1][r2] = v[r1 + A * r2];
      Dft<B, INV>::run(t[r1], tw, step);
#pragma unroll
      for (int q2 = 1; q2 < B; ++q2)
        if (r1 > 0) t[r1][q2] = cmul(t[r1][q2], tw_get<INV>(tw, r1 * q2 * step));
    }
#pragma unroll
    for (int q2 = 0; q2 < B; ++q2) {
      cf u[A];
#pragma unroll
      for (int r1 = 0; r1 < A; ++r1) u[r1] = t[r1][q2];
      Dft<A, INV>::run(u, tw, step);
#pragma unroll
      for (int q1 = 0; q1 < A; ++q1) v[q2 + B * q1] = u[q1];
    }
  }
};

template <bool INV> struct Dft<6, INV> : DftCT<2, 3, INV> {};
template <bool INV> struct Dft<8, INV> : DftCT<2, 4, INV> {};
template <bool INV> struct Dft<9, INV> : DftCT<3, 3, INV> {};
template <bool INV> struct Dft<10, INV> : DftCT<2, 5, INV> {};
template <bool INV> struct Dft<12, INV> : DftCT<3, 4, INV> {};

__host__ __device__ constexpr bool radix_ok(int r) {
  return r == 2 || r == 3 || r == 4 || r == 5 || r == 6 || r == 8 || r == 9 || r == 10 || r == 12;
}

// ---- accessors (plain structs, passed by value) -----------------------------
// element e of line l at b[l·sl + e·se]
struct Sm {
  cf* b;
  int sl, se;
  __device__ __forceinline__ cf operator()(int l, int e) const { return b[l * sl + e * se]; }
  __device__ __forceinline__ void operator()(int l, int e, cf v) const { b[l * sl + e * se] = v; }
};
struct Gm {
  cf* p;
  int64_t sl, se;
  __device__ __forceinline__ cf operator()(int l, int e) const { return p[l * sl + e * se]; }
  __device__ __forceinline__ void operator()(int l, int e, cf v) const { p[l * sl + e * se] = v; }
};

// ---- one pass ---------------------------------------------------------------
// line_fast: consecutive threads take consecutive lines (true) or consecutive
// butterflies j of one line (false).  Ends with a barrier.
template <int R, bool INV, class Ld, class St>
__device__ __forceinline__ void pass_r(const FPass& P, int nlines, unsigned Mnl, bool line_fast,
                                       const cf* tw, const Ld& ld, const St& st) {
  const int idx = threadIdx.x;
  if (idx < nlines * P.m) {
    int line, j;
    if (line_fast) {
      j = fdiv(idx, Mnl);
      line = idx - j * nlines;
    } else {
      line = fdiv(idx, P.Mm);
      j = idx - line * P.m;
    }
    cf v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = ld(line, j + r * P.m);
    int k = 0, jq = j;   // k = j mod Ns, jq = j / Ns
    if (P.Ns > 1) {
      jq = fdiv(j, P.Mns);
      k = j - jq * P.Ns;
      const int ts = k * P.twstep;
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw_get<INV>(tw, r * ts));
    }
    Dft<R, INV>::run(v, tw, P.m);
    const int base = jq * P.Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) st(line, base + r * P.Ns, v[r]);
  }
  __syncthreads();
}

template <bool INV, class Ld, class St>
__device__ __forceinline__ void pass(const FPass& P, int nlines, unsigned Mnl, bool line_fast,
                                     const cf* tw, const Ld& ld, const St& st) {
  switch (P.R) {
    case 2: pass_r<2, INV>(P, nlines, Mnl, line_fast, tw, ld, st); break;
    case 3: pass_r<3, INV>(P, nlines, Mnl, line_fast, tw, ld, st); break;
    case 4: pass_r<4, INV>(P, nlines, Mnl, line_fast, tw, ld, st); break;
    case 5: pass_r<5, INV>(P, nlines, Mnl, line_fast, tw, ld, st); break;
    case 6: pass_r<6, INV>(P, nlines, Mnl, line_fast, tw, ld, st); break;
    case 8: pass_r<8, INV>(P, nlines, Mnl, line_fast, tw, ld, st); break;
    case 9: pass_r<9, INV>(P, nlines, Mnl, line_fast, tw, ld, st); break;
    case 10: pass_r<10, INV>(P, nlines, Mnl, line_fast, tw, ld, st); break;
    case 12: pass_r<12, INV>(P, nlines, Mnl, line_fast, tw, ld, st); break;
    default: break;
  }
}

// Last forward pass fused with the first inverse pass (same radix R; forward
// Ns = n/R, inverse Ns = 1).  Thread j holds the forward outputs at j + r·m —
// exactly the inputs of inverse thread j — so fn(line, e, v) (the k-space
// mask) runs on registers in between.
template <int R, class Ld, class St, class Fn>
__device__ __forceinline__ void sandwich_r(const FPass& P, int nlines, unsigned Mnl, bool line_fast,
                                           const cf* tw, const Ld& ld, const St& st, const Fn& fn) {
  const int idx = threadIdx.x;
  const int m = P.m;
  if (idx < nlines * m) {
    int line, j;
    if (line_fast) {
      j = fdiv(idx, Mnl);
      line = idx - j * nlines;
    } else {
      line = fdiv(idx, P.Mm);
      j = idx - line * m;
    }
    cf v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = ld(line, j + r * m);
    if (m > 1) {   // forward: Ns = m, k = j, twstep = 1
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw_get<false>(tw, r * j));
    }
    Dft<R, false>::run(v, tw, m);
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = fn(line, j + r * m, v[r]);
    Dft<R, true>::run(v, tw, m);   // inverse first pass: Ns = 1, no twiddle
#pragma unroll
    for (int r = 0; r < R; ++r) st(line, j * R + r, v[r]);
  }
  __syncthreads();
}

template <class Ld, class St, class Fn>
__device__ __forceinline__ void sandwich(const FPass& P, int nlines, unsigned Mnl, bool line_fast,
                                         const cf* tw, const Ld& ld, const St& st, const Fn& fn) {
  switch (P.R) {
    case 2: sandwich_r<2>(P, nlines, Mnl, line_fast, tw, ld, st, fn); break;
    case 3: sandwich_r<3>(P, nlines, Mnl, line_fast, tw, ld, st, fn); break;
    case 4: sandwich_r<4>(P, nlines, Mnl, line_fast, tw, ld, st, fn); break;
    case 5: sandwich_r<5>(P, nlines, Mnl, line_fast, tw, ld, st, fn); break;
    case 6: sandwich_r<6>(P, nlines, Mnl, line_fast, tw, ld, st, fn); break;
    case 8: sandwich_r<8>(P, nlines, Mnl, line_fast, tw, ld, st, fn); break;
    case 9: sandwich_r<9>(P, nlines, Mnl, line_fast, tw, ld, st, fn); break;
    case 10: sandwich_r<10>(P, nlines, Mnl, line_fast, tw, ld, st, fn); break;
    case 12: sandwich_r<12>(P, nlines, Mnl, line_fast, tw, ld, st, fn); break;
    default: break;
  }
}

// Host: fill a plan from radices r[0..np) for `nlines` lines.
inline void make_fplan(int n, int np, const int* r, int nlines, FPlan* p) {
  p->n = n;
  p->npass = np;
  p->nlines = nlines;
  p->Mnl = recip(nlines);
  int Ns = 1;
  for (int i = 0; i < np; ++i) {
    FPass& P = p->fw[i];
    P.R = r[i];
    P.m = n / r[i];
    P.Ns = Ns;
    P.twstep = n / (Ns * r[i]);
    P.Mm = recip(P.m);
    P.Mns = recip(Ns);
    Ns *= r[i];
  }
  Ns = 1;
  for (int i = 0; i < np; ++i) {
    FPass& P = p->iv[i];
    const int R = r[np - 1 - i];
    P.R = R;
    P.m = n / R;
    P.Ns = Ns;
    P.twstep = n / (Ns * R);
    P.Mm = recip(P.m);
    P.Mns = recip(Ns);
    Ns *= R;
  }
}

}  // namespace fast
}  // namespace mslr
