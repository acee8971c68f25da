// fft_spec.cuh — shape-specialised FFT passes for the tuned SENSE kernels.
//
// Every axis length n = R0·R1 is a compile-time constant here, so all index
// arithmetic folds to constants, the composite butterflies' internal twiddles
// are literals (computed at compile time from a Taylor series), and each call
// site instantiates exactly one radix.
//
// Lines are owned by warps: a warp transforms LPW whole lines, lane
// (li, j) = (lane / M, lane % M) holding butterfly j of line li in a pass with
// M = n / R butterflies per line.  Because no other warp touches those lines,
// the two passes of an axis run in place in one shared buffer with only
// __syncwarp between loads and stores; block barriers are needed only where
// the line direction changes.
//
// Stockham index convention (autosort, natural order in and out), pass of
// radix R after radices of product NS, k = j mod NS, jq = j / NS:
//   in  : x[j + r·M] · w^{r·k·n/(NS·R)}
//   out : y[jq·NS·R + k + r·NS] = DFT_R(in)[r]
// Forward w = e^{−2πi/n}; the inverse is the unnormalised backward transform.
#pragma once
#include <type_traits>

#include "fft.cuh"

namespace mslr {
namespace spec {

// ---- compile-time trigonometry ----------------------------------------------
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double ct_sin(double x) {   // |x| <= π: Taylor series to double precision
  double term = x, sum = x;
  for (int i = 1; i < 40; ++i) {
    term *= -x * x / ((2.0 * i) * (2.0 * i + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double ct_cos(double x) {
  double term = 1.0, sum = 1.0;
  for (int i = 1; i < 40; ++i) {
    term *= -x * x / ((2.0 * i - 1.0) * (2.0 * i));
    sum += term;
  }
  return sum;
}

// ω_N^K = e^{∓2πiK/N} (forward −, inverse +), exact for multiples of a quarter turn
template <int N, int K, bool INV>
__device__ __forceinline__ cf cmul_w(cf v) {
  constexpr int k = ((K % N) + N) % N;
  if constexpr (k == 0) {
    return v;
  } else if constexpr (4 * k == N) {          // −i (forward)
    return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
  } else if constexpr (2 * k == N) {
    return make_float2(-v.x, -v.y);
  } else if constexpr (4 * k == 3 * N) {      // +i (forward)
    return INV ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
  } else {
    constexpr double f = (2.0 * k > N) ? (double)k / N - 1.0 : (double)k / N;
    constexpr double a = 2.0 * kPi * f;
    constexpr float c = (float)ct_cos(a);
    constexpr float s = INV ? (float)ct_sin(a) : -(float)ct_sin(a);
    return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
  }
}

template <int I, int N, class F>
__device__ __forceinline__ void sfor(F&& f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    sfor<I + 1, N>(f);
  }
}

// ---- R-point DFTs in registers ------------------------------------------------
template <int R, bool INV>
struct DK;
template <bool INV> struct DK<2, INV> { static __device__ __forceinline__ void run(cf* v) { dft2<INV>(v); } };
template <bool INV> struct DK<3, INV> { static __device__ __forceinline__ void run(cf* v) { dft3<INV>(v); } };
template <bool INV> struct DK<4, INV> { static __device__ __forceinline__ void run(cf* v) { dft4<INV>(v); } };
template <bool INV> struct DK<5, INV> { static __device__ __forceinline__ void run(cf* v) { dft5<INV>(v); } };

// R = A·B: r = r1 + A·r2, q = q2 + B·q1,
// X[q] = Σ_{r1} ω_A^{r1 q1} · ω_R^{r1 q2} · Σ_{r2} x[r1 + A r2] ω_B^{r2 q2}
template <int A, int B, bool INV>
struct DKCT {
  static __device__ __forceinline__ void run(cf* v) {
    cf t[A][B];
    sfor<0, A>([&](auto r1) {
      sfor<0, B>([&](auto r2) { t[r1][r2] = v[r1 + A * r2]; });
      DK<B, INV>::run(t[r1]);
      sfor<1, B>([&](auto q2) {
        constexpr int K = decltype(r1)::value * decltype(q2)::value;
        t[r1][q2] = cmul_w<A * B, K, INV>(t[r1][q2]);
      });
    });
    sfor<0, B>([&](auto q2) {
      cf u[A];
      sfor<0, A>([&](auto r1) { u[r1] = t[r1][q2]; });
      DK<A, INV>::run(u);
      sfor<0, A>([&](auto q1) { v[q2 + B * q1] = u[q1]; });
    });
  }
};
template <bool INV> struct DK<6, INV> : DKCT<2, 3, INV> {};
template <bool INV> struct DK<8, INV> : DKCT<2, 4, INV> {};
template <bool INV> struct DK<9, INV> : DKCT<3, 3, INV> {};
template <bool INV> struct DK<10, INV> : DKCT<2, 5, INV> {};
template <bool INV> struct DK<12, INV> : DKCT<3, 4, INV> {};
template <bool INV> struct DK<15, INV> : DKCT<3, 5, INV> {};
template <bool INV> struct DK<16, INV> : DKCT<4, 4, INV> {};

// ---- axis plans ---------------------------------------------------------------
// Two Stockham passes, forward radices (R0, R1); the inverse runs (R1, R0) so
// that the last forward and first inverse passes share radix R1.
template <int N_, int R0_, int R1_>
struct Ax2 {
  static constexpr int N = N_, R0 = R0_, R1 = R1_;
  static_assert(R0 * R1 == N, "radices must multiply to the axis length");
  static constexpr int M0 = N / R0, M1 = N / R1;
  static constexpr int MMAX = M0 > M1 ? M0 : M1;
  static_assert(MMAX <= 32, "a line's butterflies must fit one warp");
  static constexpr int LPW = 32 / MMAX;   // lines per warp
};

// ---- accessors with compile-time strides ----------------------------------------
template <int SL, int SE>
struct SmC {   // element e of line l at b[l·SL + e·SE] (shared or global)
  cf* b;
  __device__ __forceinline__ cf operator()(int l, int e) const { return b[l * SL + e * SE]; }
  __device__ __forceinline__ void operator()(int l, int e, cf v) const { b[l * SL + e * SE] = v; }
};
template <int SL>
struct GmC {   // element e of line l at p[l·SL + e·se], runtime element stride
  cf* p;
  int64_t se;
  __device__ __forceinline__ cf operator()(int l, int e) const { return p[l * SL + e * se]; }
  __device__ __forceinline__ void operator()(int l, int e, cf v) const { p[l * SL + e * se] = v; }
};

// ---- warp passes -------------------------------------------------------------------
// The lane index, re-read opaquely in every pass: the per-lane index arithmetic
// of a pass is then computed where it is used instead of being hoisted out of
// the caller's loops for every pass at once (which exhausts the registers).
__device__ __forceinline__ int opaque_lane() {
  int lane = threadIdx.x & 31;
  asm volatile("" : "+r"(lane));
  return lane;
}

// One radix-R pass of an axis of length N over lines [line0, line0 + LPW) ∩ [0, nl).
// INPLACE: loads and stores address the same buffer (a __syncwarp separates them).
// TAB: `tw` is the pass's twiddle table (build_tab), entry (r − 1)·M + j for
// butterfly j and input r — the pass must be the second of a two-pass plan
// (NS·R = N, so k = j); otherwise `tw` is the axis' e^{−2πik/N} array.
// Ends with __syncwarp, so the next pass of the same lines may read the output.
template <int N, int R, int NS, bool INV, int LPW, bool INPLACE, bool TAB = false, class Ld, class St>
__device__ __forceinline__ void wpass(int line0, int nl, const cf* tw, const Ld& ld, const St& st) {
  constexpr int M = N / R;
  constexpr int TWS = N / (NS * R);
  const int lane = opaque_lane();
  const int li = lane / M;
  const int j = lane - li * M;
  const int line = line0 + li;
  const bool act = (li < LPW) && (line < nl);
  cf v[R];
  if (act) {
    sfor<0, R>([&](auto r) { v[r] = ld(line, j + r * M); });
  }
  const int jq = j / NS, k = j - jq * NS;
  if (act) {
    if constexpr (TAB) {
      static_assert(NS * R == N, "twiddle tables serve the second pass of a two-pass plan");
      sfor<1, R>([&](auto r) { v[r] = cmul(v[r], tw_get<INV>(tw, (r - 1) * M + j)); });
    } else if constexpr (NS > 1) {
      sfor<1, R>([&](auto r) { v[r] = cmul(v[r], tw_get<INV>(tw, r * k * TWS)); });
    }
    DK<R, INV>::run(v);
  }
  if constexpr (INPLACE) __syncwarp();
  if (act) {
    const int base = jq * NS * R + k;
    sfor<0, R>([&](auto r) { st(line, base + r * NS, v[r]); });
  }
  __syncwarp();
}

// Last forward pass (radix R, NS = N/R) fused with the first inverse pass
// (radix R, NS = 1): butterfly j holds forward outputs j + r·M, exactly the
// inverse inputs, so fn(line, e, v) runs on registers in between.
// TAB: `tw` is the forward table of build_tab<N, R, N / R> (entry (r − 1)·M + j).
template <int N, int R, int LPW, bool INPLACE, bool TAB = false, class Ld, class St, class Fn>
__device__ __forceinline__ void wsandwich(int line0, int nl, const cf* tw, const Ld& ld, const St& st,
                                          const Fn& fn) {
  constexpr int M = N / R;
  const int lane = opaque_lane();
  const int li = lane / M;
  const int j = lane - li * M;
  const int line = line0 + li;
  const bool act = (li < LPW) && (line < nl);
  cf v[R];
  if (act) {
    sfor<0, R>([&](auto r) { v[r] = ld(line, j + r * M); });
    if constexpr (M > 1) {
      sfor<1, R>([&](auto r) { v[r] = cmul(v[r], tw_get<false>(tw, TAB ? (r - 1) * M + j : r * j)); });
    }
    DK<R, false>::run(v);
    sfor<0, R>([&](auto r) { v[r] = fn(line, j + r * M, v[r]); });
    DK<R, true>::run(v);
  }
  if constexpr (INPLACE) __syncwarp();
  if (act) {
    sfor<0, R>([&](auto r) { st(line, j * R + r, v[r]); });
  }
  __syncwarp();
}

// Twiddle table of the radix-R pass with M = N / R butterflies that follows a
// pass of radix M: tab[(r − 1)·M + j] = tw[r·j] for r in [1, R), j in [0, M),
// where tw[i] = e^{−2πi·i/N} (r·j < N, so the entries are exact copies).  In
// a pass, the lanes of one half-warp then read consecutive entries (lanes of
// different lines with the same j read the same one) instead of tw at
// strides r·j, which fall on few shared-memory banks.  All threads of the
// block take part; the caller synchronises before use.
template <int N, int R>
__device__ __forceinline__ void build_tab(cf* tab, const cf* __restrict__ tw) {
  constexpr int M = N / R;
  for (int i = threadIdx.x; i < (R - 1) * M; i += blockDim.x) {
    const int r = i / M + 1, j = i - (r - 1) * M;
    tab[i] = tw[r * j];
  }
}

// ---- TMA bulk copies and mbarriers -----------------------------------------------------
__device__ __forceinline__ unsigned su32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(su32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(su32(bar)), "r"(bytes)
               : "memory");
}
// Global → shared bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          su32(dst)),
      "l"(src), "r"(bytes), "r"(su32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// Shared → global bulk copy of `bytes` (multiple of 16; both addresses 16-byte
// aligned) in the issuing thread's current bulk group.
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst),
               "r"(su32(src)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// the issuing thread's bulk stores have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
// the issuing thread's bulk stores are complete (written to global memory)
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// Bounded wait for the phase of `bar` with the given parity; false on timeout.
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

}  // namespace spec
}  // namespace mslr
