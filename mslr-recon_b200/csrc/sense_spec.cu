// sense_spec.cu — shape-specialised tuned SENSE normal operator.
//
// Same decomposition as sense_fast.cu (z pass | xy pass with the k-space mask
// | z pass with the coil combine; the centring identity is in the header of
// sense.cu), compiled for the image shapes listed at the bottom of this file
// so that every axis plan, stride and line count is a compile-time constant
// (fft_spec.cuh).  The work is ordered coil group by coil group (six coils),
// two frames per chunk, so that a group's coil maps (6 × 3.9 MB at 90×90×60)
// and the chunk's k-space T (2 × 6 × 3.9 MB) stay resident in L2 together;
// the gradient g accumulates over the groups.  Per chunk:
//   k_zfwd4  persistent       Σ_k X_k · S'_c → DFT_z → T, unit (cc, f, y);
//                             coil-map slabs arrive by TMA three units ahead
//   k_xy3    persistent       plane u: DFT_x, DFT_y, mask, bDFT_y, bDFT_x;
//                             plane u + grid copied in while u is transformed
//   k_zadj5  (ch, Ny, F),     bDFT_z → × conj(S'_c), one coil per CTA, two
//            ch-CTA clusters  CTAs per SM; the cluster sums its coils through
//                             distributed shared memory in rank order
// Lines are owned by warps, so the passes of one axis need only __syncwarp;
// block barriers separate the axes and guard the copy buffers.  Every wait on
// an mbarrier is bounded: on time-out the thread stops computing, keeps
// taking part in the barriers, and the CTA raises bit 8 of the device error
// word (reported by the host after the POGM run).
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "fft_spec.cuh"
#include "internal.h"
#include "umma.cuh"

namespace cg = cooperative_groups;

namespace mslr {

namespace {

using spec::Ax2;
using spec::GmC;
using spec::SmC;

constexpr int kErrWait = kErrBulkWait;

// A copy of p the compiler cannot see through: loads through it are not
// hoisted out of the surrounding loop (which would pin every twiddle of every
// pass in registers for the whole kernel).
template <class T>
__device__ __forceinline__ T* opaque(T* p) {
  asm volatile("" : "+l"(p));
  return p;
}

template <int NX_, int NY_, int NZ_, class AX_, class AY_, class AZ_>
struct Shape {
  static constexpr int NX = NX_, NY = NY_, NZ = NZ_;
  using AX = AX_;
  using AY = AY_;
  using AZ = AZ_;
  static_assert(AX::N == NX && AY::N == NY && AZ::N == NZ, "axis plans");
  static_assert(NX % 2 == 0, "rows must be whole 16-byte units for the bulk copies");
  static constexpr int PL = NX * NY;            // plane
  static constexpr int S = NZ * NX;             // z slab (fixed y)
  static constexpr int64_t NVOX = (int64_t)PL * NZ;
  static constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }
  static constexpr int mn(int a, int b) { return a < b ? a : b; }
  static constexpr int mx(int a, int b) { return a > b ? a : b; }
  static constexpr int ZW = mn(32, cdiv(NX, AZ::LPW));                               // warps, z kernels
  // warps of the plane kernel: at most 16, so that a thread may hold 128 registers
  static constexpr int XYW = mn(16, mx(cdiv(NY, AX::LPW), cdiv(NX, AY::LPW)));
  static constexpr int MW = (PL / 32 + 2 + 3) & ~3;   // mask words spanning one plane
  static constexpr int ev(int n) { return (n + 1) & ~1; }
  // warps of the adjoint z kernel (two CTAs per SM): at most 16
  static constexpr int ZW2 = mn(16, cdiv(NX, AZ::LPW));
  // fewer warps for the z-mask kernel's third variant (more registers per
  // thread at two CTAs per SM): the most, at most 12, whose compute warps
  // divide the slab's line groups evenly (warp 0 then only moves slabs)
  static constexpr int zwm(int g) {
    int w = 12;
    while (w > 2 && g % (w - 1) != 0) --w;
    return (w > 2) ? w : mn(12, g);
  }
  static constexpr int ZWm = mn(ZW2, zwm(cdiv(NX, AZ::LPW)));
  static constexpr size_t smem_zfwd = sizeof(cf) * (4 * (size_t)S + ev(NZ)) + 3 * sizeof(uint64_t);
  static constexpr size_t smem_zadj = sizeof(cf) * (2 * (size_t)S + ev(NZ)) + sizeof(uint64_t);
  static constexpr size_t smem_xy =
      sizeof(cf) * (2 * (size_t)PL + ev(NX) + ev(NY)) + MW * sizeof(uint32_t) + sizeof(uint64_t);
  // four-pass form.  The plane kernels' work plane W (filled and read only by
  // their own passes, never by a bulk copy) has an odd row stride PW, and the
  // lines of a warp are spread over the plane (line l of group g is row or
  // column g + D·l, D = n / LPW): with NX = 90 the column passes' strided
  // accesses then fall on distinct shared-memory banks far more often than
  // with rows of 90 complex values at neighbouring lines.
  static constexpr int PW = NX | 1;
  static constexpr int spread(int n, int lpw) { return (n % lpw == 0) ? n / lpw : 0; }
  static constexpr int DC = spread(NX, AY::LPW);   // column lines (x) of the plane passes
  static constexpr int DR = spread(NY, AX::LPW);   // row lines (y)
  static constexpr size_t smem_pfwd =
      sizeof(cf) * (2 * (size_t)PL + (size_t)PW * NY + ev(NX) + ev(NY)) + sizeof(uint64_t);
  static constexpr size_t smem_zmask =
      sizeof(cf) * (2 * (size_t)S + 2 * ev(NZ)) + 8 * NZ * sizeof(uint32_t) + 2 * sizeof(uint64_t);
  static constexpr size_t smem_padj =
      sizeof(cf) * ((size_t)PL + (size_t)PW * NY + ev(NX) + ev(NY)) + sizeof(uint64_t);
};

// line l of a warp's group → row / column index (identity when D == 0)
template <int LPW, int D>
__device__ __forceinline__ int line_at(int l) {
  if constexpr (D > 0) return (l / LPW) + D * (l % LPW);
  return l;
}

// xs[z][x] · S'_c[z][x], both in shared memory (line = x, element = z)
template <int NX>
struct ZLd {
  const cf* xs;
  const cf* sc;
  __device__ __forceinline__ cf operator()(int l, int e) const {
    return cmul(xs[e * NX + l], sc[e * NX + l]);
  }
};
// dst[z][x] = conj(S'_c[z][x]) · v (in place over the k-space slab)
template <int NX>
struct ZMulC {
  cf* dst;
  const cf* sc;
  __device__ __forceinline__ void operator()(int l, int e, cf v) const {
    dst[e * NX + l] = cmulc(sc[e * NX + l], v);
  }
};
// k-space mask of one plane (line = kx, element = ky), bits staged in shared memory
template <int NX>
struct MaskS {
  const uint32_t* w;
  int off;   // bit index of (kx, ky) = (0, 0) within w
  __device__ __forceinline__ cf operator()(int l, int e, cf v) const {
    const int b = off + e * NX + l;
    return ((w[b >> 5] >> (b & 31)) & 1u) ? v : make_float2(0.f, 0.f);
  }
};

// Warp 0 copies `rows` rows of `len` complex values (row stride gs in global
// memory, dense in shared memory) and arms `bar` for the bytes.
__device__ __forceinline__ void rows_g2s(cf* dst, const cf* src, int rows, int len, int64_t gs,
                                         uint64_t* bar) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
    spec::fence_proxy_async();
    spec::mbar_expect_tx(bar, (unsigned)(rows * len * sizeof(cf)));
  }
  __syncwarp();
  for (int r = lane; r < rows; r += 32)
    spec::bulk_g2s(dst + r * len, src + r * gs, (unsigned)(len * sizeof(cf)), bar);
}

// ---------------------------------------------------------------------------
// Forward z pass of one coil group, persistent: unit u = (coil cc fastest,
// then frame, then y slab); CTA b takes the contiguous units
// [b·U/grid, (b+1)·U/grid), so the summed image slab Σ_k X_k is reloaded only
// when (y, frame) changes.  S'_c slabs arrive three units ahead by TMA; both
// passes run in place in the slab buffer; the result goes to T[f][cc][z][y][x].
template <class Sh>
__global__ void __launch_bounds__(Sh::ZW * 32, 1)
    k_zfwd4(const cf* __restrict__ X, int ns, int64_t sstride, int t0, int nf, int cc0, int ch,
            const cf* __restrict__ smod, cf* __restrict__ T, const cf* __restrict__ twz,
            int* __restrict__ err) {
  using AZ = typename Sh::AZ;
  constexpr int NX = Sh::NX, NY = Sh::NY, NZ = Sh::NZ, S = Sh::S;
  constexpr int64_t PLANE = Sh::PL, NVOX = Sh::NVOX;
  constexpr int NB = 3;
  static_assert(Sh::cdiv(NX, AZ::LPW) <= Sh::ZW, "one line group per warp");
  extern __shared__ __align__(128) unsigned char smraw[];
  cf* xs = reinterpret_cast<cf*>(smraw);
  cf* scb0 = xs + S;   // NB slab buffers
  cf* tw = scb0 + NB * S;
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw + Sh::ev(NZ));
  const int tid = threadIdx.x, warp = tid >> 5;
  const int U = NY * nf * ch;
  const int u0 = (int)((int64_t)blockIdx.x * U / gridDim.x);
  const int u1 = (int)((int64_t)(blockIdx.x + 1) * U / gridDim.x);
  if (tid == 0) {
    for (int i = 0; i < NB; ++i) spec::mbar_init(&bar[i], 1);
    spec::mbar_fence_init();
  }
  __syncthreads();
  auto issue = [&](int u, int b) {
    const int cc = u % ch, y = (u / ch) / nf;
    rows_g2s(scb0 + b * S, smod + (int64_t)(cc0 + cc) * NVOX + (int64_t)y * NX, NZ, NX, PLANE,
             &bar[b]);
  };
  if (warp == 0)
    for (int q = 0; q < NB && u0 + q < u1; ++q) issue(u0 + q, q);
  for (int i = tid; i < NZ; i += blockDim.x) tw[i] = twz[i];
  bool bad = false;
  int cur = -1;
  const int l0 = warp * AZ::LPW;
  for (int u = u0; u < u1; ++u) {
    const int q = u - u0, b = q % NB;
    const int cc = u % ch, r = u / ch, ff = r % nf, y = r / nf;
    if (r != cur) {   // new (y, frame): stage Σ_k X_k of the slab
      const int64_t base = (int64_t)(t0 + ff) * NVOX + (int64_t)y * NX;
      for (int i = tid; i < S; i += blockDim.x) {
        const int z = i / NX, x = i - z * NX;
        const int64_t off = base + z * PLANE + x;
        cf v = X[off];
        for (int k = 1; k < ns; ++k) v = cadd(v, X[off + k * sstride]);
        xs[i] = v;
      }
      cur = r;
      __syncthreads();
    }
    if (!bad && !spec::mbar_wait(&bar[b], (unsigned)((q / NB) & 1))) bad = true;
    if (!bad && l0 < NX) {
      cf* sc = scb0 + b * S;
      cf* Tc = T + ((int64_t)ff * ch + cc) * NVOX + (int64_t)y * NX;
      const cf* twc = opaque(tw);
      spec::wpass<NZ, AZ::R0, 1, false, AZ::LPW, true>(l0, NX, twc, ZLd<NX>{xs, sc},
                                                       SmC<1, NX>{sc});
      spec::wpass<NZ, AZ::R1, AZ::R0, false, AZ::LPW, false>(l0, NX, twc, SmC<1, NX>{sc},
                                                             GmC<1>{Tc, PLANE});
    }
    __syncthreads();   // slab buffer b and xs are free
    if (warp == 0 && q + NB < u1 - u0) issue(u + NB, b);
  }
  if (__syncthreads_or(bad) && tid == 0) atomicOr(err, kErrWait);
}

// The three phases of a plane, each over the lines of group l0.  Kept out of
// line so that one phase's index arithmetic is not hoisted into the plane
// loop next to the others' (which overflows the 64-register budget).
template <class Sh>
__device__ __noinline__ void xy_rows_fwd(const cf* P, cf* A, const cf* twx, int l0) {
  using AX = typename Sh::AX;
  using Rows = SmC<Sh::NX, 1>;
  spec::wpass<Sh::NX, AX::R0, 1, false, AX::LPW, false>(l0, Sh::NY, twx, Rows{const_cast<cf*>(P)},
                                                        Rows{A});
  spec::wpass<Sh::NX, AX::R1, AX::R0, false, AX::LPW, true>(l0, Sh::NY, twx, Rows{A}, Rows{A});
}
template <class Sh>
__device__ __noinline__ void xy_cols(cf* A, const cf* twy, int l0, const uint32_t* smask, int moff) {
  using AY = typename Sh::AY;
  using Cols = SmC<1, Sh::NX>;
  const MaskS<Sh::NX> msk{smask, moff};
  spec::wpass<Sh::NY, AY::R0, 1, false, AY::LPW, true>(l0, Sh::NX, twy, Cols{A}, Cols{A});
  spec::wsandwich<Sh::NY, AY::R1, AY::LPW, true>(l0, Sh::NX, twy, Cols{A}, Cols{A}, msk);
  spec::wpass<Sh::NY, AY::R0, AY::R1, true, AY::LPW, true>(l0, Sh::NX, twy, Cols{A}, Cols{A});
}
template <class Sh>
__device__ __noinline__ void xy_rows_inv(cf* A, const cf* twx, int l0, cf* pl) {
  using AX = typename Sh::AX;
  using Rows = SmC<Sh::NX, 1>;
  spec::wpass<Sh::NX, AX::R1, 1, true, AX::LPW, true>(l0, Sh::NY, twx, Rows{A}, Rows{A});
  spec::wpass<Sh::NX, AX::R0, AX::R1, true, AX::LPW, false>(l0, Sh::NY, twx, Rows{A}, Rows{pl});
}

// ---------------------------------------------------------------------------
template <class Sh>
__global__ void __launch_bounds__(Sh::XYW * 32, 1)
    k_xy3(cf* __restrict__ T, const uint32_t* __restrict__ mask, int nwords, int t0, int nf,
          int Nc, const cf* __restrict__ twx_g, const cf* __restrict__ twy_g,
          int* __restrict__ err) {
  using AX = typename Sh::AX;
  using AY = typename Sh::AY;
  constexpr int NX = Sh::NX, NY = Sh::NY, NZ = Sh::NZ, PL = Sh::PL, MW = Sh::MW;
  constexpr int64_t NVOX = Sh::NVOX;
  extern __shared__ __align__(128) unsigned char smraw[];
  cf* P = reinterpret_cast<cf*>(smraw);
  cf* A = P + PL;
  cf* twx = A + PL;
  cf* twy = twx + Sh::ev(NX);
  uint32_t* smask = reinterpret_cast<uint32_t*>(twy + Sh::ev(NY));
  uint64_t* bar = reinterpret_cast<uint64_t*>(smask + MW);
  const int tid = threadIdx.x, warp = tid >> 5, nw = blockDim.x >> 5;
  const int units = NZ * Nc * nf;
  auto plane_of = [&](int u) {
    const int kz = u % NZ, r = u / NZ;
    const int c = r % Nc, ff = r / Nc;
    return T + ((int64_t)ff * Nc + c) * NVOX + (int64_t)kz * PL;
  };
  if (tid == 0) {
    spec::mbar_init(bar, 1);
    spec::mbar_fence_init();
  }
  for (int i = tid; i < NX; i += blockDim.x) twx[i] = twx_g[i];
  for (int i = tid; i < NY; i += blockDim.x) twy[i] = twy_g[i];
  __syncthreads();
  int u = blockIdx.x;
  if (tid == 0 && u < units) {
    spec::mbar_expect_tx(bar, PL * (unsigned)sizeof(cf));
    spec::bulk_g2s(P, plane_of(u), PL * (unsigned)sizeof(cf), bar);
  }
  unsigned par = 0;
  bool bad = false;
  for (; u < units; u += gridDim.x) {
    const int kz = u % NZ, ff = u / (NZ * Nc);
    const int64_t bit0 = (int64_t)kz * PL;
    const int w0 = (int)(bit0 >> 5);
    const uint32_t* mrow = mask + (int64_t)(t0 + ff) * nwords;
    for (int i = tid; i < MW; i += blockDim.x) smask[i] = (w0 + i < nwords) ? __ldg(mrow + w0 + i) : 0u;
    if (!bad && !spec::mbar_wait(bar, par)) bad = true;
    par ^= 1u;
    if (!bad) {
#pragma unroll 1
      for (int g = warp; g * AX::LPW < NY; g += nw) xy_rows_fwd<Sh>(P, A, twx, g * AX::LPW);
    }
    __syncthreads();   // rows done; P free; mask words visible
    const int nxt = u + (int)gridDim.x;
    if (tid == 0 && nxt < units) {
      spec::fence_proxy_async();
      spec::mbar_expect_tx(bar, PL * (unsigned)sizeof(cf));
      spec::bulk_g2s(P, plane_of(nxt), PL * (unsigned)sizeof(cf), bar);
    }
    if (!bad) {
      const int moff = (int)(bit0 - (int64_t)w0 * 32);
#pragma unroll 1
      for (int g = warp; g * AY::LPW < NX; g += nw) xy_cols<Sh>(A, twy, g * AY::LPW, smask, moff);
    }
    __syncthreads();   // columns done
    if (!bad) {
      cf* pl = plane_of(u);
#pragma unroll 1
      for (int g = warp; g * AX::LPW < NY; g += nw) xy_rows_inv<Sh>(A, twx, g * AX::LPW, pl);
    }
  }
  if (__syncthreads_or(bad) && tid == 0) atomicOr(err, kErrWait);
}

// ---------------------------------------------------------------------------
// Adjoint z pass of one coil group: CTA (cc, y, f) of a cluster of `ch` CTAs
// (one per coil) takes the k-space slab of coil cc and its coil-map slab by
// TMA, runs both inverse passes in place, multiplies by conj(S'_c), and the
// cluster sums its coils through distributed shared memory in rank order into
// out (mode 0: scale·Σ − A'y when subtract, mode 1: out += scale·Σ).
template <class Sh>
__global__ void __launch_bounds__(Sh::ZW2 * 32, 2)
    k_zadj5(const cf* __restrict__ T, const cf* __restrict__ smod, cf* __restrict__ out,
            const cf* __restrict__ ahy, int t0, int cc0, float scale, int mode, int subtract,
            const cf* __restrict__ twz, int* __restrict__ err) {
  using AZ = typename Sh::AZ;
  constexpr int NX = Sh::NX, NZ = Sh::NZ, S = Sh::S;
  constexpr int64_t PLANE = Sh::PL, NVOX = Sh::NVOX;
  extern __shared__ __align__(128) unsigned char smraw[];
  cf* P = reinterpret_cast<cf*>(smraw);
  cf* SC = P + S;
  cf* tw = SC + S;
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw + Sh::ev(NZ));
  cg::cluster_group cluster = cg::this_cluster();
  const int G = (int)cluster.num_blocks();
  const int cc = (int)cluster.block_rank();
  const int tid = threadIdx.x, warp = tid >> 5, nw = blockDim.x >> 5;
  const int y = blockIdx.y, f = blockIdx.z;
  const int t = t0 + f;
  const int64_t ybase = (int64_t)y * NX;
  if (tid == 0) {
    spec::mbar_init(bar, 1);
    spec::mbar_fence_init();
  }
  __syncthreads();
  if (warp == 0) {
    const int lane = tid & 31;
    if (lane == 0) spec::mbar_expect_tx(bar, 2u * S * (unsigned)sizeof(cf));
    __syncwarp();
    const cf* ts = T + ((int64_t)f * G + cc) * NVOX + ybase;
    const cf* ss = smod + (int64_t)(cc0 + cc) * NVOX + ybase;
    for (int r = lane; r < NZ; r += 32) {
      spec::bulk_g2s(P + r * NX, ts + r * PLANE, NX * (unsigned)sizeof(cf), bar);
      spec::bulk_g2s(SC + r * NX, ss + r * PLANE, NX * (unsigned)sizeof(cf), bar);
    }
  }
  for (int i = tid; i < NZ; i += blockDim.x) tw[i] = twz[i];
  __syncthreads();
  const bool bad = !spec::mbar_wait(bar, 0);
  if (!bad) {
    const cf* twc = opaque(tw);
    using Cols = SmC<1, NX>;   // line = x, element = z
#pragma unroll 1
    for (int g = warp; g * AZ::LPW < NX; g += nw) {
      spec::wpass<NZ, AZ::R1, 1, true, AZ::LPW, true>(g * AZ::LPW, NX, twc, Cols{P}, Cols{P});
      spec::wpass<NZ, AZ::R0, AZ::R1, true, AZ::LPW, true>(g * AZ::LPW, NX, twc, Cols{P},
                                                           ZMulC<NX>{P, SC});
    }
  }
  if (__syncthreads_or(bad) && tid == 0) atomicOr(err, kErrWait);
  cluster.sync();
  // rank g sums positions [g·per, (g+1)·per) over ranks 0..G-1 in order
  const int per = (S + G - 1) / G;
  const int i0 = cc * per, i1 = min(S, i0 + per);
  for (int i = i0 + tid; i < i1; i += blockDim.x) {
    cf s = *cluster.map_shared_rank(P + i, 0);
    for (int q = 1; q < G; ++q) s = cadd(s, *cluster.map_shared_rank(P + i, q));
    const int z = i / NX, x = i - z * NX;
    const int64_t off = (int64_t)t * NVOX + z * PLANE + ybase + x;
    cf v = cscale(s, scale);
    if (mode) v = cadd(out[off], v);
    else if (subtract) v = csub(v, ahy[off]);
    out[off] = v;
  }
  cluster.sync();
}

// ===========================================================================
// Four-pass form of the normal operator (the default).  Per chunk of frames
// and group of coils, with T[f][cc][z][y][x] the chunk's per-coil k-space:
//   k_pfwd   unit (cc, z, f): S'_c ⊙ x̄ on plane z → DFT_y → DFT_x → T
//            (x̄ = Σ_k X_k, summed once per operator by k_xsum)
//   k_zmask  unit (cc, f, y): the z slab of T → DFT_z → mask → bDFT_z → T,
//            in place, slabs in and out by bulk copies
//   k_padj   unit (cc, z, f): plane of T → bDFT_y → bDFT_x → × conj(S'_c) → T
//   k_csum   g (=, −A'y, or +=) scale · Σ_cc T[f][cc], coils summed in order
// The plane passes take their planes by TMA (the next unit's while the current
// one runs its row passes); every unit is one plane or slab, so the launches
// fill all SMs evenly and no CTA waits on another.
// ===========================================================================

// x̄[i] = Σ_k X[k][i] over ns scales (in order), n elements, pairs per thread
__global__ void k_xsum(const cf* __restrict__ X, int ns, int64_t sstride, cf* __restrict__ out,
                       int64_t n) {
  const int64_t step = (int64_t)gridDim.x * blockDim.x;
  const bool vec = ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(out)) & 15) == 0 &&
                   (sstride % 2) == 0 && (n % 2) == 0;
  if (vec) {
    const float4* x4 = reinterpret_cast<const float4*>(X);
    float4* o4 = reinterpret_cast<float4*>(out);
    const int64_t n2 = n / 2, s2 = sstride / 2;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2; i += step) {
      float4 v = x4[i];
      for (int k = 1; k < ns; ++k) {
        const float4 w = x4[i + k * s2];
        v.x += w.x;
        v.y += w.y;
        v.z += w.z;
        v.w += w.w;
      }
      o4[i] = v;
    }
    return;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += step) {
    cf v = X[i];
    for (int k = 1; k < ns; ++k) v = cadd(v, X[i + k * sstride]);
    out[i] = v;
  }
}

// a[i] · b[i], both in shared memory (line l, element e at line_at(l)·SL + e·SE)
template <int SL, int SE, int LPW = 1, int D = 0>
struct LdMul {
  const cf* a;
  const cf* b;
  __device__ __forceinline__ cf operator()(int l, int e) const {
    const int i = line_at<LPW, D>(l) * SL + e * SE;
    return cmul(a[i], b[i]);
  }
};
// element e of line l at b[line_at(l)·SL + e·SE]
template <int SL, int SE, int LPW, int D>
struct SmM {
  cf* b;
  __device__ __forceinline__ cf operator()(int l, int e) const { return b[line_at<LPW, D>(l) * SL + e * SE]; }
  __device__ __forceinline__ void operator()(int l, int e, cf v) const { b[line_at<LPW, D>(l) * SL + e * SE] = v; }
};
// dst[i] = conj(s[i]) · v, row layout (line = row line_at(l), element = x); s in global memory
template <int NX, int LPW = 1, int D = 0>
struct StMulC {
  cf* dst;
  const cf* s;
  __device__ __forceinline__ void operator()(int l, int e, cf v) const {
    const int i = line_at<LPW, D>(l) * NX + e;
    dst[i] = cmulc(__ldg(s + i), v);
  }
};
// k-space mask of one z slab (line = kx, element = kz): row kz's bits start at
// bit (kz·PL + y·NX) & 31 of the four words w[4·kz ..]
template <int NX, int PL>
struct MaskZ {
  const uint32_t* w;
  int ybit;   // y·NX
  __device__ __forceinline__ cf operator()(int l, int e, cf v) const {
    const int b = ((e * PL + ybit) & 31) + l;
    return ((w[4 * e + (b >> 5)] >> (b & 31)) & 1u) ? v : make_float2(0.f, 0.f);
  }
};

// Pass groups of the plane kernels, out of line (each keeps its own index
// arithmetic, within the 128-register budget of 16 warps).  The second pass
// of each axis reads its twiddles from a table (build_tab); W has row stride
// Sh::PW and the lines of a group are spread (Sh::DC, Sh::DR).
template <class Sh>
__device__ __noinline__ void pf_cols(const cf* xs, const cf* sc, cf* W, const cf* tby, int l0) {
  using AY = typename Sh::AY;
  using Cols = SmM<1, Sh::PW, AY::LPW, Sh::DC>;
  spec::wpass<Sh::NY, AY::R0, 1, false, AY::LPW, false>(
      l0, Sh::NX, tby, LdMul<1, Sh::NX, AY::LPW, Sh::DC>{xs, sc}, Cols{W});
  spec::wpass<Sh::NY, AY::R1, AY::R0, false, AY::LPW, true, true>(l0, Sh::NX, tby, Cols{W}, Cols{W});
}
template <class Sh>
__device__ __noinline__ void pf_rows(cf* W, const cf* tbx, int l0, cf* dst) {
  using AX = typename Sh::AX;
  using Rows = SmM<Sh::PW, 1, AX::LPW, Sh::DR>;
  using Out = SmM<Sh::NX, 1, AX::LPW, Sh::DR>;
  spec::wpass<Sh::NX, AX::R0, 1, false, AX::LPW, true>(l0, Sh::NY, tbx, Rows{W}, Rows{W});
  spec::wpass<Sh::NX, AX::R1, AX::R0, false, AX::LPW, false, true>(l0, Sh::NY, tbx, Rows{W}, Out{dst});
}
template <class Sh>
__device__ __noinline__ void pa_cols(const cf* P, cf* W, const cf* tby, int l0) {
  using AY = typename Sh::AY;
  using In = SmM<1, Sh::NX, AY::LPW, Sh::DC>;
  using Cols = SmM<1, Sh::PW, AY::LPW, Sh::DC>;
  spec::wpass<Sh::NY, AY::R1, 1, true, AY::LPW, false>(l0, Sh::NX, tby, In{const_cast<cf*>(P)}, Cols{W});
  spec::wpass<Sh::NY, AY::R0, AY::R1, true, AY::LPW, true, true>(l0, Sh::NX, tby, Cols{W}, Cols{W});
}
template <class Sh>
__device__ __noinline__ void pa_rows(cf* W, const cf* tbx, int l0, cf* dst, const cf* sc) {
  using AX = typename Sh::AX;
  using Rows = SmM<Sh::PW, 1, AX::LPW, Sh::DR>;
  spec::wpass<Sh::NX, AX::R1, 1, true, AX::LPW, true>(l0, Sh::NY, tbx, Rows{W}, Rows{W});
  spec::wpass<Sh::NX, AX::R0, AX::R1, true, AX::LPW, false, true>(
      l0, Sh::NY, tbx, Rows{W}, StMulC<Sh::NX, AX::LPW, Sh::DR>{dst, sc});
}

// Forward plane pass of one coil group, persistent over units u = (cc
// fastest, then z, then frame f of the chunk): the summed image plane and the
// coil-map plane arrive by TMA; DFT_y over the columns of their product, then
// DFT_x over the rows, written to T[f][cc][z].
template <class Sh>
__global__ void __launch_bounds__(Sh::XYW * 32, 1)
    k_pfwd(const cf* __restrict__ xsum, int t0, int nf, int cc0, int ch, const cf* __restrict__ smod,
           cf* __restrict__ T, const cf* __restrict__ twx_g, const cf* __restrict__ twy_g,
           int* __restrict__ err) {
  using AX = typename Sh::AX;
  using AY = typename Sh::AY;
  constexpr int NX = Sh::NX, NY = Sh::NY, NZ = Sh::NZ, PL = Sh::PL;
  constexpr int64_t NVOX = Sh::NVOX;
  extern __shared__ __align__(128) unsigned char smraw[];
  cf* XS = reinterpret_cast<cf*>(smraw);
  cf* SB = XS + PL;
  cf* W = SB + PL;                  // row stride Sh::PW
  cf* tbx = W + Sh::PW * NY;        // twiddle tables of the second x and y passes
  cf* tby = tbx + Sh::ev(NX);
  uint64_t* bar = reinterpret_cast<uint64_t*>(tby + Sh::ev(NY));
  const int tid = threadIdx.x, warp = tid >> 5, nw = blockDim.x >> 5;
  const int units = ch * NZ * nf;
  auto issue = [&](int u) {
    const int cc = u % ch, r = u / ch, z = r % NZ, f = r / NZ;
    spec::mbar_expect_tx(bar, 2u * PL * (unsigned)sizeof(cf));
    spec::bulk_g2s(XS, xsum + (int64_t)(t0 + f) * NVOX + (int64_t)z * PL, PL * (unsigned)sizeof(cf), bar);
    spec::bulk_g2s(SB, smod + (int64_t)(cc0 + cc) * NVOX + (int64_t)z * PL, PL * (unsigned)sizeof(cf), bar);
  };
  if (tid == 0) {
    spec::mbar_init(bar, 1);
    spec::mbar_fence_init();
  }
  spec::build_tab<NX, AX::R1>(tbx, twx_g);
  spec::build_tab<NY, AY::R1>(tby, twy_g);
  __syncthreads();
  int u = blockIdx.x;
  if (tid == 0 && u < units) issue(u);
  unsigned par = 0;
  bool bad = false;
  for (; u < units; u += gridDim.x) {
    if (!bad && !spec::mbar_wait(bar, par)) bad = true;
    par ^= 1u;
    if (!bad) {
#pragma unroll 1
      for (int g = warp; g * AY::LPW < NX; g += nw) pf_cols<Sh>(XS, SB, W, tby, g * AY::LPW);
    }
    __syncthreads();   // columns done: XS, SB free
    const int nxt = u + (int)gridDim.x;
    if (tid == 0 && nxt < units) {
      spec::fence_proxy_async();
      issue(nxt);
    }
    if (!bad) {
      const int cc = u % ch, r = u / ch, z = r % NZ, f = r / NZ;
      cf* dst = T + ((int64_t)f * ch + cc) * NVOX + (int64_t)z * PL;
#pragma unroll 1
      for (int g = warp; g * AX::LPW < NY; g += nw) pf_rows<Sh>(W, tbx, g * AX::LPW, dst);
    }
    __syncthreads();   // rows done: W free
  }
  if (__syncthreads_or(bad) && tid == 0) atomicOr(err, kErrWait);
}

// z pass with the k-space mask, in place on T, persistent over slabs u = (cc
// fastest, then frame, then y): each slab (NZ rows of NX) comes in by bulk
// copies into one of two buffers, runs DFT_z, the mask and bDFT_z (the last
// forward and first inverse radix passes fused around the mask), and goes back
// by bulk copies; the other buffer's slab is in flight meanwhile.  The mask
// words of the next slab are staged (double-buffered) while the current one
// finishes, so a unit needs one block barrier.  MINB: CTAs per SM the
// register budget is set for.
template <class Sh, int MINB, int NW = Sh::ZW2>
__global__ void __launch_bounds__(NW * 32, MINB)
    k_zmask(cf* __restrict__ T, const uint32_t* __restrict__ mask, int nwords, int t0, int nf, int ch,
            const cf* __restrict__ twz_g, int* __restrict__ err) {
  using AZ = typename Sh::AZ;
  constexpr int NX = Sh::NX, NY = Sh::NY, NZ = Sh::NZ, S = Sh::S, PL = Sh::PL;
  constexpr int64_t NVOX = Sh::NVOX;
  constexpr int kGroups = Sh::cdiv(NX, AZ::LPW);   // line groups of a slab
  constexpr bool kCopyWarp = NW > 1 && kGroups % (NW - 1) == 0;
  extern __shared__ __align__(128) unsigned char smraw[];
  cf* SL = reinterpret_cast<cf*>(smraw);          // two slab buffers
  cf* tf = SL + 2 * S;                            // twiddle tables: forward (the fused pass)
  cf* ti = tf + Sh::ev(NZ);                       // and inverse (the last pass)
  uint32_t* MB = reinterpret_cast<uint32_t*>(ti + Sh::ev(NZ));   // 2 × 4 words per kz
  uint64_t* bar = reinterpret_cast<uint64_t*>(MB + 8 * NZ);
  const int tid = threadIdx.x, warp = tid >> 5, nw = blockDim.x >> 5, lane = tid & 31;
  const int units = ch * nf * NY;
  auto slab = [&](int u) {
    const int cc = u % ch, r = u / ch, f = r % nf, y = r / nf;
    return T + ((int64_t)f * ch + cc) * NVOX + (int64_t)y * NX;
  };
  if (tid == 0) {
    spec::mbar_init(&bar[0], 1);
    spec::mbar_init(&bar[1], 1);
    spec::mbar_fence_init();
  }
  // mask words of slab u into mb: row kz spans bits [kz·PL + y·NX, + NX) of frame t0 + f
  auto stage_mask = [&](int u, uint32_t* mb) {
    const int r = u / ch, f = r % nf, y = r / nf;
    const uint32_t* mrow = mask + (int64_t)(t0 + f) * nwords;
    for (int i = tid; i < 4 * NZ; i += blockDim.x) {
      const int kz = i >> 2;
      const int w = (int)(((int64_t)kz * PL + (int64_t)y * NX) >> 5) + (i & 3);
      mb[i] = (w < nwords) ? __ldg(mrow + w) : 0u;
    }
  };
  spec::build_tab<NZ, AZ::R1>(tf, twz_g);
  spec::build_tab<NZ, AZ::R0>(ti, twz_g);
  if ((int)blockIdx.x < units) stage_mask(blockIdx.x, MB);
  __syncthreads();
  if (warp == 0) {
    for (int q = 0; q < 2; ++q) {
      const int u = blockIdx.x + q * (int)gridDim.x;
      if (u < units) rows_g2s(SL + q * S, slab(u), NZ, NX, PL, &bar[q]);
    }
  }
  bool bad = false;
  int k = 0;
  for (int u = blockIdx.x; u < units; u += gridDim.x, ++k) {
    const int b = k & 1;
    const int y = (u / ch) / nf;
    if (!bad && !spec::mbar_wait(&bar[b], (unsigned)((k >> 1) & 1))) bad = true;
    cf* P = SL + b * S;
    if (!bad) {
      const cf* tfc = opaque(tf);
      const cf* tic = opaque(ti);
      using Cols = SmC<1, NX>;   // line = x, element = z
      const MaskZ<NX, PL> msk{MB + b * 4 * NZ, y * NX};
      // when the line groups divide evenly over the other warps, warp 0 only
      // moves slabs (its bulk stores and loads then overlap the others' passes)
      const int cw = kCopyWarp ? 1 : 0;
#pragma unroll 1
      for (int g = warp - cw; g >= 0 && g * AZ::LPW < NX; g += nw - cw) {
        spec::wpass<NZ, AZ::R0, 1, false, AZ::LPW, true>(g * AZ::LPW, NX, tfc, Cols{P}, Cols{P});
        spec::wsandwich<NZ, AZ::R1, AZ::LPW, true, true>(g * AZ::LPW, NX, tfc, Cols{P}, Cols{P}, msk);
        spec::wpass<NZ, AZ::R0, AZ::R1, true, AZ::LPW, true, true>(g * AZ::LPW, NX, tic, Cols{P}, Cols{P});
      }
    }
    if (u + (int)gridDim.x < units) stage_mask(u + (int)gridDim.x, MB + (b ^ 1) * 4 * NZ);
    spec::fence_proxy_async();   // this thread's slab writes, before the bulk copies read them
    __syncthreads();   // slab done; the next slab's mask words visible
    if (warp == 0) {
      if (!bad) {
        spec::fence_proxy_async();
        cf* dst = slab(u);
        for (int z = lane; z < NZ; z += 32)
          spec::bulk_s2g(dst + (int64_t)z * PL, P + z * NX, NX * (unsigned)sizeof(cf));
        spec::bulk_commit();
      }
      const int u2 = u + 2 * (int)gridDim.x;
      if (u2 < units) {
        spec::bulk_wait_read();   // this buffer's rows have left shared memory
        __syncwarp();
        rows_g2s(P, slab(u2), NZ, NX, PL, &bar[b]);
      }
    }
  }
  if (warp == 0) spec::bulk_wait_all();
  if (__syncthreads_or(bad) && tid == 0) atomicOr(err, kErrWait);
}

// Inverse plane pass, persistent over units u = (cc fastest, then z, then f):
// plane z of T[f][cc] by TMA, bDFT_y over the columns, bDFT_x over the rows,
// × conj(S'_c), written back in place.
template <class Sh>
__global__ void __launch_bounds__(Sh::XYW * 32, 1)
    k_padj(cf* __restrict__ T, int nf, int cc0, int ch, const cf* __restrict__ smod,
           const cf* __restrict__ twx_g, const cf* __restrict__ twy_g, int* __restrict__ err) {
  using AX = typename Sh::AX;
  using AY = typename Sh::AY;
  constexpr int NX = Sh::NX, NY = Sh::NY, NZ = Sh::NZ, PL = Sh::PL;
  constexpr int64_t NVOX = Sh::NVOX;
  extern __shared__ __align__(128) unsigned char smraw[];
  cf* P = reinterpret_cast<cf*>(smraw);
  cf* W = P + PL;                   // row stride Sh::PW
  cf* tbx = W + Sh::PW * NY;        // twiddle tables of the second x and y inverse passes
  cf* tby = tbx + Sh::ev(NX);
  uint64_t* bar = reinterpret_cast<uint64_t*>(tby + Sh::ev(NY));
  const int tid = threadIdx.x, warp = tid >> 5, nw = blockDim.x >> 5;
  const int units = ch * NZ * nf;
  auto plane = [&](int u) {
    const int cc = u % ch, r = u / ch, z = r % NZ, f = r / NZ;
    return T + ((int64_t)f * ch + cc) * NVOX + (int64_t)z * PL;
  };
  if (tid == 0) {
    spec::mbar_init(bar, 1);
    spec::mbar_fence_init();
  }
  spec::build_tab<NX, AX::R0>(tbx, twx_g);
  spec::build_tab<NY, AY::R0>(tby, twy_g);
  __syncthreads();
  int u = blockIdx.x;
  if (tid == 0 && u < units) {
    spec::mbar_expect_tx(bar, PL * (unsigned)sizeof(cf));
    spec::bulk_g2s(P, plane(u), PL * (unsigned)sizeof(cf), bar);
  }
  unsigned par = 0;
  bool bad = false;
  for (; u < units; u += gridDim.x) {
    if (!bad && !spec::mbar_wait(bar, par)) bad = true;
    par ^= 1u;
    if (!bad) {
#pragma unroll 1
      for (int g = warp; g * AY::LPW < NX; g += nw) pa_cols<Sh>(P, W, tby, g * AY::LPW);
    }
    __syncthreads();   // columns done: P free
    const int nxt = u + (int)gridDim.x;
    if (tid == 0 && nxt < units) {
      spec::fence_proxy_async();
      spec::mbar_expect_tx(bar, PL * (unsigned)sizeof(cf));
      spec::bulk_g2s(P, plane(nxt), PL * (unsigned)sizeof(cf), bar);
    }
    if (!bad) {
      const int cc = u % ch, z = (u / ch) % NZ;
      const cf* sc = smod + (int64_t)(cc0 + cc) * NVOX + (int64_t)z * PL;
      cf* dst = plane(u);
#pragma unroll 1
      for (int g = warp; g * AX::LPW < NY; g += nw) pa_rows<Sh>(W, tbx, g * AX::LPW, dst, sc);
    }
    __syncthreads();   // rows done: W free
  }
  if (__syncthreads_or(bad) && tid == 0) atomicOr(err, kErrWait);
}

// Coil combine of a chunk: out[t0 + f] (mode 0: scale·Σ − A'y when subtract,
// else scale·Σ; mode 1: out += scale·Σ) with Σ over the ch coils of T[f] in
// coil order.  Pairs of values per thread when every pointer is 16-byte aligned.
__global__ void k_csum(const cf* __restrict__ T, int nf, int ch, int64_t nvox, cf* __restrict__ out,
                       const cf* __restrict__ ahy, int t0, float scale, int mode, int subtract) {
  const int64_t step = (int64_t)gridDim.x * blockDim.x;
  const bool vec = ((reinterpret_cast<uintptr_t>(T) | reinterpret_cast<uintptr_t>(out) |
                     reinterpret_cast<uintptr_t>(ahy)) & 15) == 0 && (nvox % 2) == 0;
  if (vec) {
    const int64_t h = nvox / 2, n2 = (int64_t)nf * h;
    const float4* t4 = reinterpret_cast<const float4*>(T);
    float4* o4 = reinterpret_cast<float4*>(out) + (int64_t)t0 * h;
    const float4* a4 = reinterpret_cast<const float4*>(ahy) + (int64_t)t0 * h;
    if (ch == 6) {   // the compiled coil group: the six coil loads and g / A'y issued together
      for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < h; o += step) {
#pragma unroll 2
        for (int f = 0; f < nf; ++f) {
          const float4* src = t4 + (int64_t)f * 6 * h + o;
          const int64_t i = (int64_t)f * h + o;
          float4 w[6];
#pragma unroll
          for (int c = 0; c < 6; ++c) w[c] = src[c * h];
          const float4 g = mode ? o4[i] : subtract ? a4[i] : make_float4(0.f, 0.f, 0.f, 0.f);
          float4 sm = w[0];
#pragma unroll
          for (int c = 1; c < 6; ++c) {
            sm.x += w[c].x;
            sm.y += w[c].y;
            sm.z += w[c].z;
            sm.w += w[c].w;
          }
          float4 v = make_float4(sm.x * scale, sm.y * scale, sm.z * scale, sm.w * scale);
          if (mode) v = make_float4(g.x + v.x, g.y + v.y, g.z + v.z, g.w + v.w);
          else if (subtract) v = make_float4(v.x - g.x, v.y - g.y, v.z - g.z, v.w - g.w);
          o4[i] = v;
        }
      }
      return;
    }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2; i += step) {
      const int64_t f = i / h, o = i - f * h;
      const float4* src = t4 + f * ch * h + o;
      float4 s = src[0];
      for (int c = 1; c < ch; ++c) {
        const float4 w = src[c * h];
        s.x += w.x;
        s.y += w.y;
        s.z += w.z;
        s.w += w.w;
      }
      float4 v = make_float4(s.x * scale, s.y * scale, s.z * scale, s.w * scale);
      if (mode) {
        const float4 g = o4[i];
        v = make_float4(g.x + v.x, g.y + v.y, g.z + v.z, g.w + v.w);
      } else if (subtract) {
        const float4 a = a4[i];
        v = make_float4(v.x - a.x, v.y - a.y, v.z - a.z, v.w - a.w);
      }
      o4[i] = v;
    }
    return;
  }
  const int64_t n = (int64_t)nf * nvox;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += step) {
    const int64_t f = i / nvox, o = i - f * nvox;
    const cf* src = T + f * ch * nvox + o;
    cf s = src[0];
    for (int c = 1; c < ch; ++c) s = cadd(s, src[c * nvox]);
    const int64_t oi = (int64_t)t0 * nvox + i;
    cf v = cscale(s, scale);
    if (mode) v = cadd(out[oi], v);
    else if (subtract) v = csub(v, ahy[oi]);
    out[oi] = v;
  }
}

// ---------------------------------------------------------------------------
// Tensor-core plane pass (tcgen05).  The four 1-D transforms of a plane are
// dense DFT products on the tensor cores: with F[n][k] = e^{−2πi nk/N} (zero
// padded to NP, a multiple of 16) and the plane P[y][x] (y rows),
//   D1 = P F          (x forward;   A = P,    K-major, rows y)
//   D2ᵀ = D1ᵀ F       (y forward;   A = D1ᵀ,  MN-major, rows kx)
//   D3ᵀ = (M ⊙ D2)ᵀ F̄ (mask, y inverse; A K-major, rows kx)
//   D4 = D3 F̄         (x inverse;   A = D3,   MN-major, rows y)
// each a complex GEMM of M=128 × N=NP × K=NP on planar split-BF16 operands
// (hi·hi + hi·lo + lo·hi for each of the four real products; the conjugate of
// F through the negate bit), accumulated in TMEM (real and imaginary halves).
// Between products every thread takes its TMEM lane (a row of the result),
// splits it into BF16 hi / lo and writes it as the next A operand — in the
// K-major or the MN-major core-matrix layout, so no transposes are needed.
// F lives in shared memory for the whole kernel; one CTA per SM, persistent
// over the planes of the chunk.
template <int N>
struct XyT {
  static_assert(N % 2 == 0, "pairs of columns move as 16-byte vectors");
  static constexpr int NP = (N + 31) / 32 * 32;   // padded DFT length (two column halves of 16s)
  static constexpr int KC = NP / 8;               // 8-element cores per 8-row group
  static constexpr int AW = 128 * NP / 2;         // 32-bit words of a 128 × NP bf16 tile
  static constexpr int FW = NP * NP / 2;          // words of an NP × NP tile
  static constexpr unsigned SBO = KC * 128;
  static constexpr unsigned COLS = 256;           // TMEM columns: re [0, NP), im [NP, 2 NP)
  static_assert(2 * NP <= (int)COLS, "two accumulators must fit the allocation");
};

template <int N, int MW>
struct XyUSmem {
  uint32_t F[4][XyT<N>::FW];   // Fr_h, Fr_l, Fi_h, Fi_l   (K-major, row n, column k)
  uint32_t A[4][XyT<N>::AW];   // Ar_h, Ar_l, Ai_h, Ai_l
  uint32_t mask[MW];
  uint64_t bar;
  uint32_t tmem;
};

// element offset (bf16) of the first of 8 consecutive K elements (K-major) or
// 8 consecutive M elements (MN-major) of a tile with KC cores per row group
template <int KC>
__device__ __forceinline__ int kmaj8(int m, int k) { return ((m >> 3) * KC + (k >> 3)) * 64 + (m & 7) * 8; }
template <int KC>
__device__ __forceinline__ int mnmaj8(int mn, int k) { return ((mn >> 3) * KC + (k >> 3)) * 64 + (k & 7) * 8; }

// 8 complex values → 16 bytes in each of the four planar hi / lo tiles
__device__ __forceinline__ void put8(uint32_t* const* A, int eoff, const float* re, const float* im) {
  uint4 rh, rl, ih, il;
  umma::split_pair(re[0], re[1], rh.x, rl.x);
  umma::split_pair(re[2], re[3], rh.y, rl.y);
  umma::split_pair(re[4], re[5], rh.z, rl.z);
  umma::split_pair(re[6], re[7], rh.w, rl.w);
  umma::split_pair(im[0], im[1], ih.x, il.x);
  umma::split_pair(im[2], im[3], ih.y, il.y);
  umma::split_pair(im[4], im[5], ih.z, il.z);
  umma::split_pair(im[6], im[7], ih.w, il.w);
  const int w = eoff >> 1;
  *reinterpret_cast<uint4*>(A[0] + w) = rh;
  *reinterpret_cast<uint4*>(A[1] + w) = rl;
  *reinterpret_cast<uint4*>(A[2] + w) = ih;
  *reinterpret_cast<uint4*>(A[3] + w) = il;
}

// one complex DFT product into TMEM (issued by one thread): A (MN-major when
// AMN) times F (forward) or conj(F) (INV)
template <int N, int MW, bool AMN, bool INV>
__device__ __forceinline__ void dft_gemm(const XyUSmem<N, MW>& s, uint32_t dre, uint32_t dim) {
  using X = XyT<N>;
  constexpr uint32_t P = umma::idesc(128, X::NP, false, false, AMN, false);
  constexpr uint32_t Ng = umma::idesc(128, X::NP, true, false, AMN, false);
#pragma unroll 1
  for (int t = 0; t < X::NP / 16; ++t) {
    auto a = [&](int i) { return umma::sdesc(s.A[i] + t * 64, 128, X::SBO); };
    auto f = [&](int i) { return umma::sdesc(s.F[i] + t * 64, 128, X::SBO); };
    const bool acc = t > 0;
    // Re += Ar·Fr ∓ Ai·Fi      (forward: −, inverse: +)
    umma::mma(dre, a(0), f(0), P, acc);
    umma::mma(dre, a(0), f(1), P, true);
    umma::mma(dre, a(1), f(0), P, true);
    umma::mma(dre, a(2), f(2), INV ? P : Ng, true);
    umma::mma(dre, a(2), f(3), INV ? P : Ng, true);
    umma::mma(dre, a(3), f(2), INV ? P : Ng, true);
    // Im += ±Ar·Fi + Ai·Fr     (forward: +, inverse: −)
    umma::mma(dim, a(0), f(2), INV ? Ng : P, acc);
    umma::mma(dim, a(0), f(3), INV ? Ng : P, true);
    umma::mma(dim, a(1), f(2), INV ? Ng : P, true);
    umma::mma(dim, a(2), f(0), P, true);
    umma::mma(dim, a(2), f(1), P, true);
    umma::mma(dim, a(3), f(0), P, true);
  }
}

template <class Sh>
__global__ void __launch_bounds__(256, 1)
    k_xy_umma(cf* __restrict__ T, const uint32_t* __restrict__ mask, int nwords, int t0, int nf,
              int Nc, const uint32_t* __restrict__ Fg, int* __restrict__ err) {
  static_assert(Sh::NX == Sh::NY, "square planes");
  constexpr int N = Sh::NX, NZ = Sh::NZ, PL = Sh::PL, MW = Sh::MW;
  constexpr int64_t NVOX = Sh::NVOX;
  using X = XyT<N>;
  using Sm = XyUSmem<N, MW>;
  constexpr int NP = X::NP, KC = X::KC;
  extern __shared__ __align__(1024) unsigned char smraw[];
  Sm& s = *reinterpret_cast<Sm*>(smraw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row = (warp & 3) * 32 + lane;   // TMEM lane of this thread
  const int half = warp >> 2;              // column half of the epilogues
  // DFT matrix into shared memory, operand tile cleared (rows >= NP stay zero)
  for (int i = tid; i < 4 * X::FW / 4; i += 256)
    reinterpret_cast<uint4*>(&s.F[0][0])[i] = __ldg(reinterpret_cast<const uint4*>(Fg) + i);
  for (int i = tid; i < 4 * X::AW / 4; i += 256)
    reinterpret_cast<uint4*>(&s.A[0][0])[i] = make_uint4(0u, 0u, 0u, 0u);
  umma::tmem_alloc(&s.tmem, X::COLS);
  if (tid == 0) {
    umma::mbar_init(&s.bar);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  umma::fence_after();
  const uint32_t tm = s.tmem;
  const uint32_t lane_addr = tm + ((uint32_t)((warp & 3) * 32) << 16);
  uint32_t* Aarr[4] = {s.A[0], s.A[1], s.A[2], s.A[3]};
  const int units = NZ * Nc * nf;
  unsigned phase = 0;
  bool ok = true;
  // one GEMM: make the operand visible, issue, wait; false on time-out
  auto run = [&](auto amn, auto inv) {
    umma::fence_async_smem();
    umma::fence_before();
    __syncthreads();
    if (tid == 0 && ok) {
      umma::fence_after();
      dft_gemm<N, MW, decltype(amn)::value, decltype(inv)::value>(s, tm, tm + NP);
      umma::commit(&s.bar);
    }
    if (ok && !umma::mbar_wait(&s.bar, phase)) ok = false;
    phase ^= 1u;
    ok = __syncthreads_and(ok);
    umma::fence_after();
  };
  using F_ = std::false_type;
  using T_ = std::true_type;
  for (int u = blockIdx.x; u < units && ok; u += gridDim.x) {
    const int kz = u % NZ, r = u / NZ;
    const int c = r % Nc, ff = r / Nc;
    cf* pl = T + ((int64_t)ff * Nc + c) * NVOX + (int64_t)kz * PL;
    const int64_t bit0 = (int64_t)kz * PL;
    const int w0 = (int)(bit0 >> 5);
    const int moff = (int)(bit0 - (int64_t)w0 * 32);
    const uint32_t* mrow = mask + (int64_t)(t0 + ff) * nwords;
    for (int i = tid; i < MW; i += 256) s.mask[i] = (w0 + i < nwords) ? __ldg(mrow + w0 + i) : 0u;
    // E0: plane rows → A (K-major, m = y, k = x)
    if (row < NP) {
      for (int cb = 0; cb < NP / 32; ++cb) {
        const int c0 = half * (NP / 2) + cb * 16;
        float re[16], im[16];
#pragma unroll
        for (int j = 0; j < 16; j += 2) {
          const int x = c0 + j;
          float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
          if (row < N && x < N) v = __ldg(reinterpret_cast<const float4*>(pl + row * N + x));
          re[j] = v.x;
          im[j] = v.y;
          re[j + 1] = v.z;
          im[j + 1] = v.w;
        }
        put8(Aarr, kmaj8<KC>(row, c0), re, im);
        put8(Aarr, kmaj8<KC>(row, c0 + 8), re + 8, im + 8);
      }
    }
    run(F_{}, F_{});   // D1 = P F: lanes y, columns kx
    // E1: D1 → A (MN-major, mn = kx, k = y)
    for (int cb = 0; cb < NP / 32; ++cb) {
      const int c0 = half * (NP / 2) + cb * 16;
      float re[16], im[16];
      umma::ld16(lane_addr + c0, re);
      umma::ld16(lane_addr + NP + c0, im);
      if (row < NP) {
        put8(Aarr, mnmaj8<KC>(c0, row), re, im);
        put8(Aarr, mnmaj8<KC>(c0 + 8, row), re + 8, im + 8);
      }
    }
    run(T_{}, F_{});   // D2ᵀ: lanes kx, columns ky
    // E2: mask, → A (K-major, m = kx, k = ky)
    for (int cb = 0; cb < NP / 32; ++cb) {
      const int c0 = half * (NP / 2) + cb * 16;
      float re[16], im[16];
      umma::ld16(lane_addr + c0, re);
      umma::ld16(lane_addr + NP + c0, im);
      if (row < NP) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int ky = c0 + j;
          bool keep = false;
          if (row < N && ky < N) {
            const int b = moff + ky * N + row;
            keep = (s.mask[b >> 5] >> (b & 31)) & 1u;
          }
          if (!keep) re[j] = im[j] = 0.f;
        }
        put8(Aarr, kmaj8<KC>(row, c0), re, im);
        put8(Aarr, kmaj8<KC>(row, c0 + 8), re + 8, im + 8);
      }
    }
    run(F_{}, T_{});   // D3ᵀ: lanes kx, columns y
    // E3: → A (MN-major, mn = y, k = kx)
    for (int cb = 0; cb < NP / 32; ++cb) {
      const int c0 = half * (NP / 2) + cb * 16;
      float re[16], im[16];
      umma::ld16(lane_addr + c0, re);
      umma::ld16(lane_addr + NP + c0, im);
      if (row < NP) {
        put8(Aarr, mnmaj8<KC>(c0, row), re, im);
        put8(Aarr, mnmaj8<KC>(c0 + 8, row), re + 8, im + 8);
      }
    }
    run(T_{}, T_{});   // D4: lanes y, columns x
    // E4: → plane rows in global memory
    for (int cb = 0; cb < NP / 32; ++cb) {
      const int c0 = half * (NP / 2) + cb * 16;
      float re[16], im[16];
      umma::ld16(lane_addr + c0, re);
      umma::ld16(lane_addr + NP + c0, im);
      if (row < N) {
#pragma unroll
        for (int j = 0; j < 16; j += 2) {
          const int x = c0 + j;
          if (x < N) *reinterpret_cast<float4*>(pl + row * N + x) = make_float4(re[j], im[j], re[j + 1], im[j + 1]);
        }
      }
    }
    umma::fence_before();
    __syncthreads();   // plane done: A and the mask words may be rewritten
  }
  if (__syncthreads_or(!ok) && tid == 0) atomicOr(err, kErrWait);
  umma::tmem_free(tm, X::COLS);
}

// F[n][k] = e^{−2πi nk/N}, zero padded to NP × NP, as the four split-BF16
// K-major tiles of k_xy_umma (host, double precision before the split)
template <int N>
std::vector<uint32_t> dft_tiles() {
  using X = XyT<N>;
  constexpr int NP = X::NP, KC = X::KC;
  std::vector<uint16_t> t(4 * (size_t)NP * NP, 0);
  auto bf = [](float v) {   // round to nearest even
    uint32_t b;
    std::memcpy(&b, &v, 4);
    return (uint16_t)((b + 0x7FFFu + ((b >> 16) & 1u)) >> 16);
  };
  auto fl = [](uint16_t h) {
    const uint32_t b = (uint32_t)h << 16;
    float v;
    std::memcpy(&v, &b, 4);
    return v;
  };
  for (int n = 0; n < N; ++n)
    for (int k = 0; k < N; ++k) {
      const double a = -2.0 * 3.14159265358979323846 * (double)((int64_t)n * k % N) / N;
      const float re = (float)std::cos(a), im = (float)std::sin(a);
      const uint16_t rh = bf(re), ih = bf(im);
      const uint16_t rl = bf(re - fl(rh)), il = bf(im - fl(ih));
      const size_t e = (size_t)((n >> 3) * KC + (k >> 3)) * 64 + (n & 7) * 8 + (k & 7);
      t[0 * (size_t)NP * NP + e] = rh;
      t[1 * (size_t)NP * NP + e] = rl;
      t[2 * (size_t)NP * NP + e] = ih;
      t[3 * (size_t)NP * NP + e] = il;
    }
  std::vector<uint32_t> w(t.size() / 2);
  std::memcpy(w.data(), t.data(), t.size() * sizeof(uint16_t));
  return w;
}

// ---------------------------------------------------------------------------
struct SpecOps {
  int nx, ny, nz;
  const void* zfwd;
  const void* xy;
  const void* zadj;
  int zfwd_threads, xy_threads, zadj_threads;
  size_t smem_zfwd, smem_zadj, smem_xy;
  // four-pass form
  const void* pfwd;
  const void* zmask;     // two CTAs per SM (64 registers)
  const void* zmask1;    // one CTA per SM (more registers, MSLR_ZMASK_CTAS=1)
  const void* zmaskm;    // two CTAs per SM with Sh::ZWm warps (more registers per thread)
  int zmaskm_threads;
  const void* padj;
  size_t smem_pfwd, smem_zmask, smem_padj;
  const void* xy_tc;                       // tensor-core plane pass (square planes), or null
  size_t smem_xy_tc;
  std::vector<uint32_t> (*dft)();          // its DFT tiles
};

template <class Sh>
SpecOps ops_of() {
  SpecOps o{Sh::NX,
            Sh::NY,
            Sh::NZ,
            reinterpret_cast<const void*>(&k_zfwd4<Sh>),
            reinterpret_cast<const void*>(&k_xy3<Sh>),
            reinterpret_cast<const void*>(&k_zadj5<Sh>),
            Sh::ZW * 32,
            Sh::XYW * 32,
            Sh::ZW2 * 32,
            Sh::smem_zfwd,
            Sh::smem_zadj,
            Sh::smem_xy,
            reinterpret_cast<const void*>(&k_pfwd<Sh>),
            reinterpret_cast<const void*>(&k_zmask<Sh, 2>),
            reinterpret_cast<const void*>(&k_zmask<Sh, 1>),
            reinterpret_cast<const void*>(&k_zmask<Sh, 2, Sh::ZWm>),
            Sh::ZWm * 32,
            reinterpret_cast<const void*>(&k_padj<Sh>),
            Sh::smem_pfwd,
            Sh::smem_zmask,
            Sh::smem_padj,
            nullptr,
            0,
            nullptr};
  if constexpr (Sh::NX == Sh::NY && Sh::NX <= 128) {
    o.xy_tc = reinterpret_cast<const void*>(&k_xy_umma<Sh>);
    o.smem_xy_tc = sizeof(XyUSmem<Sh::NX, Sh::MW>);
    o.dft = &dft_tiles<Sh::NX>;
  }
  return o;
}

// Compiled shapes: the reference's fMRI volume (90×90×60) and smaller cubes
// used by its tests and synthetic studies.
using S90 = Shape<90, 90, 60, Ax2<90, 10, 9>, Ax2<90, 10, 9>, Ax2<60, 10, 6>>;
using S48 = Shape<48, 48, 32, Ax2<48, 8, 6>, Ax2<48, 8, 6>, Ax2<32, 8, 4>>;
using S32 = Shape<32, 32, 24, Ax2<32, 8, 4>, Ax2<32, 8, 4>, Ax2<24, 6, 4>>;

const SpecOps* find_ops(int nx, int ny, int nz) {
  static const SpecOps table[] = {ops_of<S90>(), ops_of<S48>(), ops_of<S32>()};
  for (const SpecOps& o : table)
    if (o.nx == nx && o.ny == ny && o.nz == nz) return &o;
  return nullptr;
}

}  // namespace

bool sense_spec_setup(Ctx* c) {
  const SpecOps* o = find_ops(c->N[0], c->N[1], c->N[2]);
  if (!o) return false;
  if (cudaFuncSetAttribute(o->zfwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)o->smem_zfwd) ||
      cudaFuncSetAttribute(o->zadj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)o->smem_zadj) ||
      cudaFuncSetAttribute(o->xy, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)o->smem_xy)) {
    cudaGetLastError();
    return false;
  }
  int per_sm = 0, per_sm_z = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, o->xy, o->xy_threads, o->smem_xy) ||
      per_sm < 1 ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_z, o->zfwd, o->zfwd_threads,
                                                    o->smem_zfwd) ||
      per_sm_z < 1) {
    cudaGetLastError();
    return false;
  }
  int dev = 0, nsm = 0;
  if (!cudaGetDevice(&dev) && !cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) &&
      nsm > 0)
    c->nsm = nsm;
  cudaGetLastError();
  c->spec_xy_ctas = per_sm * c->nsm;
  // chunk shape (the autotuner may refine it): 6 coils per group, and the most
  // frames per chunk (up to 4) for which the chunk's k-space and the group's
  // coil maps, (frames + 1) · 6 images, stay within about 120 MB of the L2
  c->spec_ch = 6;
  {
    const double img = (double)c->nvox * sizeof(cf);
    int fr = 4;
    while (fr > 1 && (double)std::min(c->Nc, 6) * (fr + 1) * img > 120e6) --fr;
    c->spec_fr = fr;
  }
  c->spec_zfwd_ctas = per_sm_z * c->nsm;
  // four-pass form (default; MSLR_SENSE_PATH=3 keeps the three-kernel form)
  {
    const char* sp = std::getenv("MSLR_SENSE_PATH");
    c->spec_four = !(sp && std::string(sp) == "3");
  }
  if (c->spec_four) {
    const char* zc = std::getenv("MSLR_ZMASK_CTAS");
    c->spec_zmask_var = (zc && std::string(zc) == "1") ? 1 : 0;
    int a = 0, b = 0, b1 = 0, bm = 0, d = 0;
    if (cudaFuncSetAttribute(o->pfwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)o->smem_pfwd) ||
        cudaFuncSetAttribute(o->zmask, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)o->smem_zmask) ||
        cudaFuncSetAttribute(o->zmask1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)o->smem_zmask) ||
        cudaFuncSetAttribute(o->zmaskm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)o->smem_zmask) ||
        cudaFuncSetAttribute(o->padj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)o->smem_padj) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, o->pfwd, o->xy_threads, o->smem_pfwd) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, o->zmask, o->zadj_threads, o->smem_zmask) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, o->zmask1, o->zadj_threads, o->smem_zmask) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bm, o->zmaskm, o->zmaskm_threads, o->smem_zmask) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, o->padj, o->xy_threads, o->smem_padj) ||
        a < 1 || b < 1 || b1 < 1 || bm < 1 || d < 1 ||
        dalloc(c, (void**)&c->d_xsum, (size_t)c->Nt * c->nvox * sizeof(cf))) {
      cudaGetLastError();
      c->spec_four = false;
    } else {
      c->spec_pfwd_ctas = a * c->nsm;
      c->spec_zmask_ctas_v[0] = b * c->nsm;
      c->spec_zmask_ctas_v[1] = b1 * c->nsm;
      c->spec_zmask_ctas_v[2] = bm * c->nsm;
      c->spec_zmask_warps[0] = c->spec_zmask_warps[1] = o->zadj_threads / 32;
      c->spec_zmask_warps[2] = o->zmaskm_threads / 32;
      c->spec_zmask_ctas = c->spec_zmask_ctas_v[c->spec_zmask_var];
      c->spec_padj_ctas = d * c->nsm;
      // two lanes by default (measured 8.65 → 7.77 ms for a 40-frame operator
      // at 90×90×60 × 18 coils); MSLR_SENSE_LANES=1 keeps one
      const char* ln = std::getenv("MSLR_SENSE_LANES");
      if (!(ln && std::string(ln) == "1") &&
          !cudaStreamCreateWithFlags(&c->sn_stream, cudaStreamNonBlocking) &&
          !cudaEventCreateWithFlags(&c->sn_fork, cudaEventDisableTiming) &&
          !cudaEventCreateWithFlags(&c->sn_join, cudaEventDisableTiming))
        c->spec_lanes = 2;
      cudaGetLastError();
    }
  }
  // tensor-core plane pass only on request (MSLR_XY_PATH=tc): at 90×90 its
  // padded split-BF16 DFT products (12 MMAs of 128×96×16 per K step, four
  // products per plane, serialised with their epilogues) take longer than the
  // FP32 FFT plane pass
  const char* xp = std::getenv("MSLR_XY_PATH");
  c->xy_tc = false;
  if (o->xy_tc && xp && std::string(xp) == "tc" && o->smem_xy_tc <= 227 * 1024 &&
      !cudaFuncSetAttribute(o->xy_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)o->smem_xy_tc)) {
    const std::vector<uint32_t> t = o->dft();
    if (!c->d_dft && !dalloc(c, (void**)&c->d_dft, t.size() * sizeof(uint32_t)) &&
        !cudaMemcpy(c->d_dft, t.data(), t.size() * sizeof(uint32_t), cudaMemcpyHostToDevice))
      c->xy_tc = true;
  }
  cudaGetLastError();
  return true;
}

// Records a profiling event on st when the context is profiling.
static int prof_mark(Ctx* c, cudaStream_t st) {
  if (!c->prof_on) return MSLR_OK;
  if (c->prof_n == (int)c->prof_ev.size()) {
    cudaEvent_t e;
    MSLR_CUDA_TRY(cudaEventCreate(&e));
    c->prof_ev.push_back(e);
  }
  MSLR_CUDA_TRY(cudaEventRecord(c->prof_ev[c->prof_n++], st));
  return MSLR_OK;
}

// Four-pass normal operator (see k_pfwd ... k_csum): Σ_k X_k once, then per
// coil group and chunk of frames the four kernels; consecutive chunks
// alternate between two streams ("lanes", each with its own k-space buffer),
// so that one chunk's memory-bound coil combine and its kernels' last waves
// overlap the next chunk's kernels.
static int normal_op_four(Ctx* c, const SpecOps* o, const cf* X, int ns, int64_t sstride, cf* g,
                          bool subtract, cudaStream_t st) {
  const float scale = (float)(1.0 / (double)c->nvox);
  const int Nc = c->Nc;
  const int Ch = std::max(1, std::min(Nc, c->spec_ch));             // coils per group
  int F = std::max(1, c->spec_fr);                                  // frames per chunk
  while (F > 1 && (int64_t)F * Ch > (int64_t)c->F * Nc) --F;        // within the k-space buffer
  const int64_t nvox = c->nvox;
  // the summed image: X itself for one 16-byte aligned image, else Σ_k X_k
  const cf* xs = X;
  if (ns > 1 || (reinterpret_cast<uintptr_t>(X) & 15)) {
    k_xsum<<<4 * c->nsm, 512, 0, st>>>(X, ns, sstride, c->d_xsum, (int64_t)c->Nt * nvox);
    MSLR_CUDA_TRY(cudaGetLastError());
    c->launches += 1;
    xs = c->d_xsum;
  }
  int nwords = c->nwords;
  const cf* smod = c->d_smaps_mod;
  const uint32_t* mask = c->d_mask;
  const cf* ahy = c->d_ahy;
  cf* T = c->d_T;
  int* err = c->d_err;
  const int sub = subtract ? 1 : 0;
  const int zv = c->spec_zmask_var;
  const void* zk = zv == 1 ? o->zmask1 : zv == 2 ? o->zmaskm : o->zmask;
  const int zthreads = zv == 2 ? o->zmaskm_threads : o->zadj_threads;
  c->prof_kernels = 4;
  // two lanes: chunk j of every group on lane j % 2 (so the += of later
  // groups stays ordered after the first group's chunk of the same frames),
  // each lane with its own k-space buffer
  const int64_t chunk_imgs = (int64_t)F * Ch;
  const bool lanes = c->spec_lanes == 2 && !c->prof_on && 2 * chunk_imgs <= (int64_t)c->F * Nc &&
                     c->Nt > F;
  cudaStream_t side = c->sn_stream;
  if (lanes) {
    MSLR_CUDA_TRY(cudaEventRecord(c->sn_fork, st));
    MSLR_CUDA_TRY(cudaStreamWaitEvent(side, c->sn_fork, 0));
  }
  cudaStream_t st0 = st;
  for (int cc0 = 0; cc0 < Nc; cc0 += Ch) {
    int ch = std::min(Ch, Nc - cc0);
    const int mode = cc0 > 0 ? 1 : 0;
    for (int t0 = 0, j = 0; t0 < c->Nt; t0 += F, ++j) {
      int f = std::min(F, c->Nt - t0);
      const int lane = lanes ? (j & 1) : 0;
      st = lane ? side : st0;
      T = c->d_T + lane * chunk_imgs * nvox;
      const int planes = ch * c->N[2] * f;
      if (int rc = prof_mark(c, st)) return rc;
      {
        const int grid = std::max(1, std::min(planes, c->spec_pfwd_ctas));
        void* args[] = {(void*)&xs, (void*)&t0, (void*)&f, (void*)&cc0, (void*)&ch, (void*)&smod,
                        (void*)&T,  (void*)&c->d_tw[0], (void*)&c->d_tw[1], (void*)&err};
        MSLR_CUDA_TRY(cudaLaunchKernel(o->pfwd, dim3(grid), dim3(o->xy_threads), args, o->smem_pfwd, st));
      }
      if (int rc = prof_mark(c, st)) return rc;
      {
        const int slabs = ch * f * c->N[1];
        const int grid = std::max(1, std::min(slabs, c->spec_zmask_ctas));
        void* args[] = {(void*)&T, (void*)&mask, (void*)&nwords, (void*)&t0, (void*)&f, (void*)&ch,
                        (void*)&c->d_tw[2], (void*)&err};
        MSLR_CUDA_TRY(cudaLaunchKernel(zk, dim3(grid), dim3(zthreads), args, o->smem_zmask, st));
      }
      if (int rc = prof_mark(c, st)) return rc;
      {
        const int grid = std::max(1, std::min(planes, c->spec_padj_ctas));
        void* args[] = {(void*)&T,  (void*)&f, (void*)&cc0, (void*)&ch, (void*)&smod,
                        (void*)&c->d_tw[0], (void*)&c->d_tw[1], (void*)&err};
        MSLR_CUDA_TRY(cudaLaunchKernel(o->padj, dim3(grid), dim3(o->xy_threads), args, o->smem_padj, st));
      }
      if (int rc = prof_mark(c, st)) return rc;
      k_csum<<<4 * c->nsm, 512, 0, st>>>(T, f, ch, nvox, g, ahy, t0, scale, mode, sub);
      MSLR_CUDA_TRY(cudaGetLastError());
      if (int rc = prof_mark(c, st)) return rc;
      c->launches += 4;
    }
  }
  if (lanes) {   // join the side lane back into the caller's stream
    MSLR_CUDA_TRY(cudaEventRecord(c->sn_join, side));
    MSLR_CUDA_TRY(cudaStreamWaitEvent(st0, c->sn_join, 0));
  }
  return MSLR_OK;
}

int normal_op_spec(Ctx* c, const cf* X, int ns, int64_t sstride, cf* g, bool subtract,
                   cudaStream_t st) {
  const SpecOps* o = find_ops(c->N[0], c->N[1], c->N[2]);
  if (!o) return fail(MSLR_ERR_UNSUPPORTED, "no specialised SENSE kernels for this shape");
  if (c->spec_four && !c->xy_tc) return normal_op_four(c, o, X, ns, sstride, g, subtract, st);
  c->prof_kernels = 3;
  float scale = (float)(1.0 / (double)c->nvox);
  const int Nc = c->Nc, Ny = c->N[1], Nz = c->N[2];
  const int Ch = std::max(1, std::min(Nc, c->spec_ch));             // coils per group
  int F = std::max(1, c->spec_fr);                                  // frames per chunk
  while (F > 1 && (int64_t)F * Ch > (int64_t)c->F * Nc) --F;        // within the k-space buffer
  int nwords = c->nwords;
  const cf* smod = c->d_smaps_mod;
  const uint32_t* mask = c->d_mask;
  const cf* ahy = c->d_ahy;
  cf* T = c->d_T;
  int* err = c->d_err;
  int sub = subtract ? 1 : 0;
  for (int cc0 = 0; cc0 < Nc; cc0 += Ch) {
    int ch = std::min(Ch, Nc - cc0);
    int mode = cc0 > 0 ? 1 : 0;
    for (int t0 = 0; t0 < c->Nt; t0 += F) {
      int f = std::min(F, c->Nt - t0);
      if (int rc = prof_mark(c, st)) return rc;
      {
        const int U = Ny * f * ch;
        const int grid = std::max(1, std::min(U, c->spec_zfwd_ctas));
        void* args[] = {(void*)&X,  (void*)&ns,   (void*)&sstride, (void*)&t0,
                        (void*)&f,  (void*)&cc0,  (void*)&ch,      (void*)&smod,
                        (void*)&T,  (void*)&c->d_tw[2], (void*)&err};
        MSLR_CUDA_TRY(cudaLaunchKernel(o->zfwd, dim3(grid), dim3(o->zfwd_threads), args,
                                       o->smem_zfwd, st));
      }
      if (int rc = prof_mark(c, st)) return rc;
      if (c->xy_tc) {
        const int units = Nz * ch * f;
        const int grid = std::max(1, std::min(units, c->nsm));
        const uint32_t* dft = c->d_dft;
        void* args[] = {(void*)&T,  (void*)&mask, (void*)&nwords, (void*)&t0, (void*)&f,
                        (void*)&ch, (void*)&dft,  (void*)&err};
        MSLR_CUDA_TRY(cudaLaunchKernel(o->xy_tc, dim3(grid), dim3(256), args, o->smem_xy_tc, st));
      } else {
        const int units = Nz * ch * f;
        const int grid = std::max(1, std::min(units, c->spec_xy_ctas));
        void* args[] = {(void*)&T,  (void*)&mask,       (void*)&nwords,      (void*)&t0, (void*)&f,
                        (void*)&ch, (void*)&c->d_tw[0], (void*)&c->d_tw[1], (void*)&err};
        MSLR_CUDA_TRY(
            cudaLaunchKernel(o->xy, dim3(grid), dim3(o->xy_threads), args, o->smem_xy, st));
      }
      if (int rc = prof_mark(c, st)) return rc;
      {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(ch, Ny, f);
        cfg.blockDim = dim3(o->zadj_threads, 1, 1);
        cfg.dynamicSmemBytes = o->smem_zadj;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = ch;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        const cf* Tc = T;
        void* args[] = {(void*)&Tc,   (void*)&smod, (void*)&g,   (void*)&ahy,
                        (void*)&t0,   (void*)&cc0,  (void*)&scale, (void*)&mode,
                        (void*)&sub,  (void*)&c->d_tw[2], (void*)&err};
        MSLR_CUDA_TRY(cudaLaunchKernelExC(&cfg, o->zadj, args));
      }
      if (int rc = prof_mark(c, st)) return rc;
      c->launches += 3;
    }
  }
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

// Autotuner: coils per group × frames per chunk of the specialised normal
// operator, timed on the bound context (A'A applied to A'y).  Larger chunks
// mean fewer launches; the chunk's k-space (Ch·F images) and the group's coil
// maps should stay in L2.  Clusters of the adjoint z kernel hold Ch CTAs, so
// Ch ≤ 8.
int tune_sense_chunks(Ctx* c, cudaStream_t st) {
  if (!c->spec) return MSLR_OK;
  // the three-kernel form's clusters hold one coil per CTA (at most 8); the
  // four-pass form takes any group size
  const bool four = c->spec_four && !c->xy_tc;
  std::vector<int> chs = {2, 3, 4, 6, 8};
  if (four) chs.insert(chs.end(), {9, 12, 18});
  const int64_t E = (int64_t)c->Nt * c->nvox;
  float best = 1e30f;
  int bch = c->spec_ch, bfr = c->spec_fr;
  for (int ch : chs) {
    if (ch > c->Nc) continue;
    for (int fr = 1; fr <= 4; ++fr) {
      if ((int64_t)fr * ch > (int64_t)c->F * c->Nc || fr > c->Nt || fr * ch > 24) continue;
      c->spec_ch = ch;
      c->spec_fr = fr;
      float ms = 0.f;
      int rc = time_ms(st, 2, &ms, [&] { return normal_op_spec(c, c->d_ahy, 1, E, c->d_G, false, st); });
      if (rc) return rc;
      if (ms < best) {
        best = ms;
        bch = ch;
        bfr = fr;
      }
    }
  }
  c->spec_ch = bch;
  c->spec_fr = bfr;
  return MSLR_OK;
}

// Autotuner, four-pass form: one or two lanes (streams) for the chunks, and
// the z-mask kernel variant — two CTAs per SM (64 registers), one CTA per SM
// (more registers, fewer slabs in flight), or two CTAs per SM of fewer warps
// (more registers per thread) — timed on the chosen chunk shape.
int tune_sense_variants(Ctx* c, cudaStream_t st) {
  if (!c->spec || !c->spec_four || c->xy_tc) return MSLR_OK;
  const int64_t E = (int64_t)c->Nt * c->nvox;
  const int max_lanes = c->sn_stream ? 2 : 1;
  float best = 1e30f;
  int bl = c->spec_lanes, bz = c->spec_zmask_var;
  for (int lanes = 1; lanes <= max_lanes; ++lanes) {
    for (int z1 = 0; z1 <= 2; ++z1) {
      c->spec_lanes = lanes;
      c->spec_zmask_var = z1;
      c->spec_zmask_ctas = c->spec_zmask_ctas_v[z1];
      float ms = 0.f;
      int rc = time_ms(st, 2, &ms, [&] { return normal_op_spec(c, c->d_ahy, 1, E, c->d_G, false, st); });
      if (rc) return rc;
      if (ms < best) {
        best = ms;
        bl = lanes;
        bz = z1;
      }
    }
  }
  c->spec_lanes = bl;
  c->spec_zmask_var = bz;
  c->spec_zmask_ctas = c->spec_zmask_ctas_v[bz];
  return MSLR_OK;
}

int autotune(Ctx* c, cudaStream_t st) {
  int rc = tune_sense_chunks(c, st);
  if (!rc) rc = tune_sense_variants(c, st);
  if (!rc) rc = tune_svst_splits(c, st);
  if (!rc) rc = tune_eig_variants(c, st);
  if (c->gexec) {   // the captured iteration holds the old launch shapes
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
    c->gX = nullptr;
  }
  return rc;
}

}  // namespace mslr
