// sense_fast.cu — tuned SENSE normal operator (and forward / adjoint).
//
// Same mathematics and decomposition as sense.cu (z pass, xy pass, z pass with
// coil combine; see the header of sense.cu for the centring identity), built
// from the register-resident passes of fft_fast.cuh:
//   k_zfwd_fast  grid (G, Ny, F)   Σ_k X_k → × S'_c → DFT_z, G coil groups
//   k_xy_fast    grid (Nz, Nc, F)  DFT_x, DFT_y, mask, bDFT_y, bDFT_x on one
//                                  plane; the mask is applied in registers
//                                  between the last forward and the first
//                                  inverse y pass
//   k_zadj_fast  grid (G, Ny, F)   bDFT_z → × conj(S'_c), accumulated per coil
//                                  group in shared memory and reduced across
//                                  a G-CTA cluster through distributed shared
//                                  memory in a fixed rank order
// The first pass of every kernel reads global memory directly and the last
// pass writes it directly.  One frame per chunk keeps the per-coil k-space of
// the chunk (Nc × Nvox × 8 bytes, 70 MB at 90×90×60×18) resident in L2.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

#include "fft_fast.cuh"
#include "internal.h"

namespace cg = cooperative_groups;

namespace mslr {

using fast::FPass;
using fast::FPlan;
using fast::Gm;
using fast::Sm;

namespace {

constexpr int kThreads = fast::kMaxThreads;

struct Dims {
  int Nx, Ny, Nz, Nc;
  int64_t nvox;
};

enum XyMode { XY_NORMAL = 0, XY_FORWARD = 1, XY_ADJOINT = 2 };

__device__ __forceinline__ void load_tw(cf* dst, const cf* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// Passes [p0, p1) of ps.  When gf, pass p0 reads through ldf and writes `a`;
// otherwise the data start in `a`.  SMEM-to-SMEM passes alternate a/b.  When
// gl, pass p1-1 writes through stl.  Returns the buffer holding the data
// (meaningless when gl).
template <bool INV, class LdF, class StL>
__device__ __forceinline__ Sm run_passes(const FPass* ps, int p0, int p1, int nl, unsigned Mnl,
                                         bool lf, const cf* tw, const LdF& ldf, const StL& stl,
                                         bool gf, bool gl, Sm a, Sm b) {
  Sm cur = a, oth = b;
  for (int p = p0; p < p1; ++p) {
    const bool first = gf && p == p0, last = gl && p == p1 - 1;
    if (first && last) {
      fast::pass<INV>(ps[p], nl, Mnl, lf, tw, ldf, stl);
    } else if (first) {
      fast::pass<INV>(ps[p], nl, Mnl, lf, tw, ldf, cur);
    } else if (last) {
      fast::pass<INV>(ps[p], nl, Mnl, lf, tw, cur, stl);
    } else {
      fast::pass<INV>(ps[p], nl, Mnl, lf, tw, cur, oth);
      const Sm t = cur;
      cur = oth;
      oth = t;
    }
  }
  return cur;
}

// z-slab accessors (line = x, element = z) ------------------------------------
struct ZLoadMul {   // xs[z][x] · S'_c[z][y][x]
  const cf* xs;
  const cf* sc;
  int Nx;
  int64_t plane;
  __device__ __forceinline__ cf operator()(int l, int e) const {
    return cmul(xs[e * Nx + l], sc[e * plane + l]);
  }
};
struct ZAcc {       // acc[z][x] += conj(S'_c[z][y][x]) · v
  cf* acc;
  const cf* sc;
  int Nx;
  int64_t plane;
  __device__ __forceinline__ void operator()(int l, int e, cf v) const {
    cf& a = acc[e * Nx + l];
    a = cadd(a, cmulc(sc[e * plane + l], v));
  }
};
struct MaskFn {     // keep k-space samples of frame t: plane kz, (kx = l, ky = e)
  const uint32_t* mk;
  int64_t kbase;
  int Nx;
  __device__ __forceinline__ cf operator()(int l, int e, cf v) const {
    const int64_t k = kbase + (int64_t)e * Nx + l;
    return ((__ldg(mk + (k >> 5)) >> (k & 31)) & 1u) ? v : make_float2(0.f, 0.f);
  }
};

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1)
    k_zfwd_fast(const cf* __restrict__ X, int ns, int64_t sstride, int t0,
                const cf* __restrict__ smod, cf* __restrict__ T, Dims d, FPlan pz,
                const cf* __restrict__ twz, int cpg) {
  extern __shared__ cf sm[];
  const int S = d.Nz * d.Nx;
  cf* tw = sm;
  cf* xs = tw + d.Nz;
  cf* A = xs + S;
  cf* B = A + S;   // used only by three-pass plans
  const int grp = blockIdx.x, y = blockIdx.y, f = blockIdx.z;
  const int t = t0 + f;
  load_tw(tw, twz, d.Nz);
  const int64_t plane = (int64_t)d.Nx * d.Ny;
  const int64_t ybase = (int64_t)y * d.Nx;
  for (int i = threadIdx.x; i < S; i += blockDim.x) {
    const int z = i / d.Nx, x = i - z * d.Nx;
    const int64_t off = (int64_t)t * d.nvox + z * plane + ybase + x;
    cf v = X[off];
    for (int k = 1; k < ns; ++k) v = cadd(v, X[off + k * sstride]);
    xs[i] = v;
  }
  __syncthreads();
  const int c0 = grp * cpg, c1 = min(d.Nc, c0 + cpg);
  const Sm sa{A, 1, d.Nx}, sb{B, 1, d.Nx};
  for (int c = c0; c < c1; ++c) {
    const ZLoadMul ldf{xs, smod + (int64_t)c * d.nvox + ybase, d.Nx, plane};
    const Gm stl{T + ((int64_t)f * d.Nc + c) * d.nvox + ybase, 1, plane};
    run_passes<false>(pz.fw, 0, pz.npass, d.Nx, pz.Mnl, true, tw, ldf, stl, true, true, sa, sb);
  }
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1)
    k_xy_fast(cf* __restrict__ T, const uint32_t* __restrict__ mask, int nwords, int t0, Dims d,
              FPlan px, FPlan py, const cf* __restrict__ twx_g, const cf* __restrict__ twy_g,
              int mode) {
  extern __shared__ cf sm[];
  const int P = d.Nx * d.Ny;
  const int Nx = d.Nx, Ny = d.Ny;
  cf* twx = sm;
  cf* twy = twx + Nx;
  cf* A = twy + Ny;
  cf* B = A + P;
  const int kz = blockIdx.x, c = blockIdx.y, f = blockIdx.z;
  const int t = t0 + f;
  load_tw(twx, twx_g, Nx);
  load_tw(twy, twy_g, Ny);
  __syncthreads();
  cf* pl = T + ((int64_t)f * d.Nc + c) * d.nvox + (int64_t)kz * P;
  const Gm grow{pl, Nx, 1};   // x axis: line = row y, element = x
  const Gm gcol{pl, 1, Nx};   // y axis: line = column x, element = y
  auto rows = [&](cf* b) { return Sm{b, Nx, 1}; };
  auto cols = [&](cf* b) { return Sm{b, 1, Nx}; };
  auto other = [&](const cf* b) { return b == A ? B : A; };
  if (mode == XY_NORMAL) {
    Sm cur = run_passes<false>(px.fw, 0, px.npass, Ny, px.Mnl, false, twx, grow, grow, true,
                               false, rows(A), rows(B));
    cur = run_passes<false>(py.fw, 0, py.npass - 1, Nx, py.Mnl, true, twy, gcol, gcol, false,
                            false, cols(cur.b), cols(other(cur.b)));
    const Sm dst = cols(other(cur.b));
    const MaskFn msk{mask + (int64_t)t * nwords, (int64_t)kz * P, Nx};
    fast::sandwich(py.fw[py.npass - 1], Nx, py.Mnl, true, twy, cols(cur.b), dst, msk);
    cur = run_passes<true>(py.iv, 1, py.npass, Nx, py.Mnl, true, twy, gcol, gcol, false, false,
                           dst, cols(other(dst.b)));
    run_passes<true>(px.iv, 0, px.npass, Ny, px.Mnl, false, twx, grow, grow, false, true,
                     rows(cur.b), rows(other(cur.b)));
  } else if (mode == XY_FORWARD) {
    Sm cur = run_passes<false>(px.fw, 0, px.npass, Ny, px.Mnl, false, twx, grow, grow, true,
                               false, rows(A), rows(B));
    run_passes<false>(py.fw, 0, py.npass, Nx, py.Mnl, true, twy, gcol, gcol, false, true,
                      cols(cur.b), cols(other(cur.b)));
  } else {
    Sm cur = run_passes<true>(py.iv, 0, py.npass, Nx, py.Mnl, true, twy, gcol, gcol, true, false,
                              cols(A), cols(B));
    run_passes<true>(px.iv, 0, px.npass, Ny, px.Mnl, false, twx, grow, grow, false, true,
                     rows(cur.b), rows(other(cur.b)));
  }
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1)
    k_zadj_fast(const cf* __restrict__ T, const cf* __restrict__ smod, cf* __restrict__ out,
                const cf* __restrict__ ahy, int t0, float scale, int subtract, Dims d, FPlan pz,
                const cf* __restrict__ twz, int cpg) {
  extern __shared__ cf sm[];
  const int S = d.Nz * d.Nx;
  cf* tw = sm;
  cf* acc = tw + d.Nz;
  cf* A = acc + S;
  cf* B = A + S;   // used only by three-pass plans
  cg::cluster_group cluster = cg::this_cluster();
  const int G = (int)cluster.num_blocks();
  const int grp = (int)cluster.block_rank();
  const int y = blockIdx.y, f = blockIdx.z;
  const int t = t0 + f;
  load_tw(tw, twz, d.Nz);
  for (int i = threadIdx.x; i < S; i += blockDim.x) acc[i] = make_float2(0.f, 0.f);
  __syncthreads();
  const int64_t plane = (int64_t)d.Nx * d.Ny;
  const int64_t ybase = (int64_t)y * d.Nx;
  const int c0 = grp * cpg, c1 = min(d.Nc, c0 + cpg);
  const Sm sa{A, 1, d.Nx}, sb{B, 1, d.Nx};
  for (int c = c0; c < c1; ++c) {
    const Gm ldf{const_cast<cf*>(T) + ((int64_t)f * d.Nc + c) * d.nvox + ybase, 1, plane};
    // each output position is owned by one thread for every coil: no race on acc
    const ZAcc stl{acc, smod + (int64_t)c * d.nvox + ybase, d.Nx, plane};
    run_passes<true>(pz.iv, 0, pz.npass, d.Nx, pz.Mnl, true, tw, ldf, stl, true, true, sa, sb);
  }
  cluster.sync();
  // rank g reduces positions [g·per, (g+1)·per) over ranks 0..G-1 in order
  const int per = (S + G - 1) / G;
  const int i0 = grp * per, i1 = min(S, i0 + per);
  for (int i = i0 + (int)threadIdx.x; i < i1; i += blockDim.x) {
    cf s = *cluster.map_shared_rank(acc + i, 0);
    for (int q = 1; q < G; ++q) s = cadd(s, *cluster.map_shared_rank(acc + i, q));
    const int z = i / d.Nx, x = i - z * d.Nx;
    const int64_t off = (int64_t)t * d.nvox + z * plane + ybase + x;
    cf v = cscale(s, scale);
    if (subtract) v = csub(v, ahy[off]);
    out[off] = v;
  }
  cluster.sync();
}

// ---- prefetching variants ----------------------------------------------------
// Shared-memory slabs arrive by cp.async while the previous coil or plane is
// being transformed, so the global latency of a CTA's inputs is paid once.

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// dst[r·len + e] = src[r·gs + e], r < rows, e < len
__device__ __forceinline__ void slab_async(cf* dst, const cf* src, int rows, int len, int64_t gs) {
  const int tot = rows * len;
  for (int i = threadIdx.x; i < tot; i += blockDim.x) {
    const int r = i / len, e = i - r * len;
    cp_async8(dst + i, src + r * gs + e);
  }
}
// dst[i] = src[i], i < cnt (16-byte copies when both ends allow it)
__device__ __forceinline__ void span_async(cf* dst, const cf* src, int cnt) {
  const bool v16 = ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15) == 0;
  if (v16) {
    const int h = cnt >> 1;
    for (int i = threadIdx.x; i < h; i += blockDim.x) cp_async16(dst + 2 * i, src + 2 * i);
    if ((cnt & 1) && threadIdx.x == 0) cp_async8(dst + cnt - 1, src + cnt - 1);
  } else {
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) cp_async8(dst + i, src + i);
  }
}

struct ZLoadMulS {   // xs[z][x] · S'_c[z][x], both staged in shared memory
  const cf* xs;
  const cf* sc;
  int Nx;
  __device__ __forceinline__ cf operator()(int l, int e) const {
    return cmul(xs[e * Nx + l], sc[e * Nx + l]);
  }
};
struct ZAccS {       // acc[z][x] += conj(S'_c[z][x]) · v, S'_c staged in shared memory
  cf* acc;
  const cf* sc;
  int Nx;
  __device__ __forceinline__ void operator()(int l, int e, cf v) const {
    cf& a = acc[e * Nx + l];
    a = cadd(a, cmulc(sc[e * Nx + l], v));
  }
};

// k_zfwd_fast with the coil-map slab of the next coil prefetched.
// Shared: tw[Nz], xs, sc, A (, B for three-pass plans), each Nz·Nx.
__global__ void __launch_bounds__(kThreads, 1)
    k_zfwd_pre(const cf* __restrict__ X, int ns, int64_t sstride, int t0,
               const cf* __restrict__ smod, cf* __restrict__ T, Dims d, FPlan pz,
               const cf* __restrict__ twz, int cpg) {
  extern __shared__ __align__(16) cf sm[];
  const int S = d.Nz * d.Nx;
  cf* tw = sm;
  cf* xs = tw + ((d.Nz + 1) & ~1);
  cf* sc = xs + S;
  cf* A = sc + S;
  cf* B = A + S;
  const int grp = blockIdx.x, y = blockIdx.y, f = blockIdx.z;
  const int t = t0 + f;
  const int64_t plane = (int64_t)d.Nx * d.Ny;
  const int64_t ybase = (int64_t)y * d.Nx;
  const int c0 = grp * cpg, c1 = min(d.Nc, c0 + cpg);
  if (c0 < c1) slab_async(sc, smod + (int64_t)c0 * d.nvox + ybase, d.Nz, d.Nx, plane);
  cp_commit();
  load_tw(tw, twz, d.Nz);
  for (int i = threadIdx.x; i < S; i += blockDim.x) {
    const int z = i / d.Nx, x = i - z * d.Nx;
    const int64_t off = (int64_t)t * d.nvox + z * plane + ybase + x;
    cf v = X[off];
    for (int k = 1; k < ns; ++k) v = cadd(v, X[off + k * sstride]);
    xs[i] = v;
  }
  const Sm sa{A, 1, d.Nx}, sb{B, 1, d.Nx};
  const ZLoadMulS ldf{xs, sc, d.Nx};
  for (int c = c0; c < c1; ++c) {
    cp_wait_all();
    __syncthreads();
    const Gm stl{T + ((int64_t)f * d.Nc + c) * d.nvox + ybase, 1, plane};
    if (pz.npass == 1) {
      fast::pass<false>(pz.fw[0], d.Nx, pz.Mnl, true, tw, ldf, stl);
    } else {
      fast::pass<false>(pz.fw[0], d.Nx, pz.Mnl, true, tw, ldf, sa);
    }
    if (c + 1 < c1) slab_async(sc, smod + (int64_t)(c + 1) * d.nvox + ybase, d.Nz, d.Nx, plane);
    cp_commit();
    if (pz.npass > 1)
      run_passes<false>(pz.fw, 1, pz.npass, d.Nx, pz.Mnl, true, tw, sa, stl, false, true, sa, sb);
  }
}

// k_zadj_fast with the next coil's k-space slab and coil-map slab prefetched.
// Shared: tw[Nz], acc, A, P, SC0, SC1 (, B for three-pass plans), each Nz·Nx.
__global__ void __launch_bounds__(kThreads, 1)
    k_zadj_pre(const cf* __restrict__ T, const cf* __restrict__ smod, cf* __restrict__ out,
               const cf* __restrict__ ahy, int t0, float scale, int subtract, Dims d, FPlan pz,
               const cf* __restrict__ twz, int cpg) {
  extern __shared__ __align__(16) cf sm[];
  const int S = d.Nz * d.Nx;
  cf* tw = sm;
  cf* acc = tw + ((d.Nz + 1) & ~1);
  cf* A = acc + S;
  cf* P = A + S;
  cf* SC0 = P + S;
  cf* SC1 = SC0 + S;
  cf* B = SC1 + S;
  cg::cluster_group cluster = cg::this_cluster();
  const int G = (int)cluster.num_blocks();
  const int grp = (int)cluster.block_rank();
  const int y = blockIdx.y, f = blockIdx.z;
  const int t = t0 + f;
  const int64_t plane = (int64_t)d.Nx * d.Ny;
  const int64_t ybase = (int64_t)y * d.Nx;
  const int c0 = grp * cpg, c1 = min(d.Nc, c0 + cpg);
  auto tslab = [&](int c) { return T + ((int64_t)f * d.Nc + c) * d.nvox + ybase; };
  if (c0 < c1) {
    slab_async(P, tslab(c0), d.Nz, d.Nx, plane);
    slab_async(SC0, smod + (int64_t)c0 * d.nvox + ybase, d.Nz, d.Nx, plane);
  }
  cp_commit();
  load_tw(tw, twz, d.Nz);
  for (int i = threadIdx.x; i < S; i += blockDim.x) acc[i] = make_float2(0.f, 0.f);
  const Sm sa{A, 1, d.Nx}, sb{B, 1, d.Nx}, sp{P, 1, d.Nx};
  for (int c = c0; c < c1; ++c) {
    cp_wait_all();
    __syncthreads();
    const int q = c - c0;
    // each output position is owned by one thread for every coil: no race on acc
    const ZAccS stl{acc, (q & 1) ? SC1 : SC0, d.Nx};
    if (pz.npass == 1) {
      fast::pass<true>(pz.iv[0], d.Nx, pz.Mnl, true, tw, sp, stl);
    } else {
      fast::pass<true>(pz.iv[0], d.Nx, pz.Mnl, true, tw, sp, sa);
    }
    if (c + 1 < c1) {
      slab_async(P, tslab(c + 1), d.Nz, d.Nx, plane);
      slab_async((q & 1) ? SC0 : SC1, smod + (int64_t)(c + 1) * d.nvox + ybase, d.Nz, d.Nx, plane);
    }
    cp_commit();
    if (pz.npass > 1)
      run_passes<true>(pz.iv, 1, pz.npass, d.Nx, pz.Mnl, true, tw, sa, stl, false, true, sa, sb);
  }
  cluster.sync();
  // rank g reduces positions [g·per, (g+1)·per) over ranks 0..G-1 in order
  const int per = (S + G - 1) / G;
  const int i0 = grp * per, i1 = min(S, i0 + per);
  for (int i = i0 + (int)threadIdx.x; i < i1; i += blockDim.x) {
    cf s = *cluster.map_shared_rank(acc + i, 0);
    for (int q = 1; q < G; ++q) s = cadd(s, *cluster.map_shared_rank(acc + i, q));
    const int z = i / d.Nx, x = i - z * d.Nx;
    const int64_t off = (int64_t)t * d.nvox + z * plane + ybase + x;
    cf v = cscale(s, scale);
    if (subtract) v = csub(v, ahy[off]);
    out[off] = v;
  }
  cluster.sync();
}

// Persistent normal-mode plane kernel: CTA b takes planes b, b + grid, ...
// (plane u = kz + Nz·(c + Nc·f)); the next plane is copied into P while the
// current one is transformed in A / B.  Shared: twx, twy, P, A, B.
__global__ void __launch_bounds__(kThreads, 1)
    k_xy_pers(cf* __restrict__ T, const uint32_t* __restrict__ mask, int nwords, int t0, int nf,
              Dims d, FPlan px, FPlan py, const cf* __restrict__ twx_g,
              const cf* __restrict__ twy_g) {
  extern __shared__ __align__(16) cf sm[];
  const int Pl = d.Nx * d.Ny;
  const int Nx = d.Nx, Ny = d.Ny;
  cf* twx = sm;
  cf* twy = twx + Nx;
  cf* P = twy + ((Ny + 1) & ~1) + (Nx & 1);   // 16-byte aligned when sm is
  cf* A = P + ((Pl + 1) & ~1);
  cf* B = A + ((Pl + 1) & ~1);
  const int units = d.Nz * d.Nc * nf;
  auto plane_of = [&](int u) {
    const int kz = u % d.Nz, r = u / d.Nz;
    const int c = r % d.Nc, ff = r / d.Nc;
    return T + ((int64_t)ff * d.Nc + c) * d.nvox + (int64_t)kz * Pl;
  };
  int u = blockIdx.x;
  if (u < units) span_async(P, plane_of(u), Pl);
  cp_commit();
  load_tw(twx, twx_g, Nx);
  load_tw(twy, twy_g, Ny);
  auto rows = [&](cf* b) { return Sm{b, Nx, 1}; };
  auto cols = [&](cf* b) { return Sm{b, 1, Nx}; };
  auto other = [&](const cf* b) { return b == A ? B : A; };
  for (; u < units; u += gridDim.x) {
    cp_wait_all();
    __syncthreads();
    const int kz = u % d.Nz, ff = u / (d.Nz * d.Nc);
    cf* pl = plane_of(u);
    const Gm grow{pl, Nx, 1};
    fast::pass<false>(px.fw[0], Ny, px.Mnl, false, twx, rows(P), rows(A));
    const int nxt = u + (int)gridDim.x;
    if (nxt < units) span_async(P, plane_of(nxt), Pl);
    cp_commit();
    Sm cur = run_passes<false>(px.fw, 1, px.npass, Ny, px.Mnl, false, twx, grow, grow, false,
                               false, rows(A), rows(B));
    cur = run_passes<false>(py.fw, 0, py.npass - 1, Nx, py.Mnl, true, twy, grow, grow, false,
                            false, cols(cur.b), cols(other(cur.b)));
    const Sm dst = cols(other(cur.b));
    const MaskFn msk{mask + (int64_t)(t0 + ff) * nwords, (int64_t)kz * Pl, Nx};
    fast::sandwich(py.fw[py.npass - 1], Nx, py.Mnl, true, twy, cols(cur.b), dst, msk);
    cur = run_passes<true>(py.iv, 1, py.npass, Nx, py.Mnl, true, twy, grow, grow, false, false,
                           dst, cols(other(dst.b)));
    run_passes<true>(px.iv, 0, px.npass, Ny, px.Mnl, false, twx, grow, grow, false, true,
                     rows(cur.b), rows(other(cur.b)));
  }
}

// y[t][c][i] = s·φ(idx)·T[f][c][idx]  /  its adjoint scatter
__device__ __forceinline__ cf phase_at(int64_t k, const cf* px, const cf* py, const cf* pz,
                                       const Dims& d) {
  const int x = (int)(k % d.Nx);
  const int y = (int)((k / d.Nx) % d.Ny);
  const int z = (int)(k / ((int64_t)d.Nx * d.Ny));
  return cmul(px[x], cmul(py[y], pz[z]));
}

__global__ void k_gather_fast(const cf* __restrict__ T, const int32_t* __restrict__ idx,
                              cf* __restrict__ yout, int t0, int64_t K, float s, const cf* px,
                              const cf* py, const cf* pz, Dims d) {
  const int c = blockIdx.y, f = blockIdx.z;
  const int t = t0 + f;
  const cf* Tc = T + ((int64_t)f * d.Nc + c) * d.nvox;
  const int32_t* it = idx + (int64_t)t * K;
  cf* yo = yout + ((int64_t)t * d.Nc + c) * K;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < K;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = it[i];
    yo[i] = cscale(cmul(phase_at(k, px, py, pz, d), Tc[k]), s);
  }
}

__global__ void k_scatter_fast(cf* __restrict__ T, const int32_t* __restrict__ idx,
                               const cf* __restrict__ yin, int t0, int64_t K, float s,
                               const cf* px, const cf* py, const cf* pz, Dims d) {
  const int c = blockIdx.y, f = blockIdx.z;
  const int t = t0 + f;
  cf* Tc = T + ((int64_t)f * d.Nc + c) * d.nvox;
  const int32_t* it = idx + (int64_t)t * K;
  const cf* yi = yin + ((int64_t)t * d.Nc + c) * K;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < K;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = it[i];
    Tc[k] = cscale(cmulc(phase_at(k, px, py, pz, d), yi[i]), s);
  }
}

Dims dims_of(const Ctx* c) {
  Dims d;
  d.Nx = c->N[0];
  d.Ny = c->N[1];
  d.Nz = c->N[2];
  d.Nc = c->Nc;
  d.nvox = c->nvox;
  return d;
}

size_t smem_z(const Ctx* c, int npass) {
  const size_t S = (size_t)c->N[2] * c->N[0];
  return sizeof(cf) * (c->N[2] + (npass >= 3 ? 3 : 2) * S);
}
size_t smem_xy(const Ctx* c) {
  return sizeof(cf) * (c->N[0] + c->N[1] + 2 * (size_t)c->N[0] * c->N[1]);
}
size_t smem_zfwd_pre(const Ctx* c, int npass) {
  const size_t S = (size_t)c->N[2] * c->N[0];
  return sizeof(cf) * (((c->N[2] + 1) & ~1) + (npass >= 3 ? 4 : 3) * S);
}
size_t smem_zadj_pre(const Ctx* c, int npass) {
  const size_t S = (size_t)c->N[2] * c->N[0];
  return sizeof(cf) * (((c->N[2] + 1) & ~1) + (npass >= 3 ? 6 : 5) * S);
}
size_t smem_xy_pers(const Ctx* c) {
  const size_t Pl = (size_t)c->N[0] * c->N[1];
  return sizeof(cf) * (c->N[0] + ((c->N[1] + 1) & ~1) + (c->N[0] & 1) + 3 * ((Pl + 1) & ~1));
}

// Radices (1-3 passes, every radix in the menu, at most kThreads butterflies
// per pass for `nl` lines).  Prefers two balanced radices.
bool choose_radices(int n, int nl, int* np, int* r) {
  auto ok = [&](int R) { return fast::radix_ok(R) && (int64_t)nl * (n / R) <= kThreads; };
  if (n >= 2 && ok(n)) {
    *np = 1;
    r[0] = n;
    return true;
  }
  int b0 = 0, b1 = 0;
  for (int a = 2; a <= 12; ++a) {
    if (n % a) continue;
    const int b = n / a;
    if (!ok(a) || !ok(b)) continue;
    if (std::min(a, b) > std::min(b0, b1) || (std::min(a, b) == std::min(b0, b1) && a > b0)) {
      b0 = a;
      b1 = b;
    }
  }
  if (b0) {
    *np = 2;
    r[0] = b0;
    r[1] = b1;
    return true;
  }
  for (int a = 2; a <= 12; ++a)
    for (int b = 2; b <= 12; ++b) {
      if (n % (a * b)) continue;
      const int cc = n / (a * b);
      if (ok(a) && ok(b) && ok(cc)) {
        *np = 3;
        r[0] = a;
        r[1] = b;
        r[2] = cc;
        return true;
      }
    }
  return false;
}

int groups_of(int Nc) { return std::min(Nc, 6); }

}  // namespace

// Plans for the tuned kernels; false when the image shape needs the generic path.
bool sense_fast_setup(Ctx* c) {
  const int Nx = c->N[0], Ny = c->N[1], Nz = c->N[2];
  int np[3], r[3][3];
  if (!choose_radices(Nx, Ny, &np[0], r[0]) || !choose_radices(Ny, Nx, &np[1], r[1]) ||
      !choose_radices(Nz, Nx, &np[2], r[2]))
    return false;
  if (Nx >= 1024 || Ny >= 1024 || Nz >= 1024) return false;
  FPlan* fp = reinterpret_cast<FPlan*>(c->fplan_raw);
  static_assert(sizeof(FPlan) * 3 <= sizeof(c->fplan_raw), "fplan storage");
  fast::make_fplan(Nx, np[0], r[0], Ny, &fp[0]);
  fast::make_fplan(Ny, np[1], r[1], Nx, &fp[1]);
  fast::make_fplan(Nz, np[2], r[2], Nx, &fp[2]);
  const size_t sz = smem_z(c, np[2]), sxy = smem_xy(c);
  if (sz > 200 * 1024 || sxy > 200 * 1024) return false;
  if (raise_dyn_smem((const void*)k_zfwd_fast, (int)sz) ||
      raise_dyn_smem((const void*)k_zadj_fast, (int)sz) ||
      raise_dyn_smem((const void*)k_xy_fast, (int)sxy)) {
    cudaGetLastError();
    return false;
  }
  // prefetching variants where their extra buffers fit
  constexpr size_t kMaxSmem = 227 * 1024;
  const size_t szf = smem_zfwd_pre(c, np[2]), sza = smem_zadj_pre(c, np[2]), sxp = smem_xy_pers(c);
  c->zpre = szf <= kMaxSmem && sza <= kMaxSmem &&
            !raise_dyn_smem((const void*)k_zfwd_pre, (int)szf) &&
            !raise_dyn_smem((const void*)k_zadj_pre, (int)sza);
  c->xypers = sxp <= kMaxSmem &&
              !raise_dyn_smem((const void*)k_xy_pers, (int)sxp);
  cudaGetLastError();
  int dev = 0, nsm = 0;
  if (!cudaGetDevice(&dev) && !cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) && nsm > 0)
    c->nsm = nsm;
  cudaGetLastError();
  return true;
}

namespace {

int launch_zadj(Ctx* c, const Dims& d, int G, int f, int t0, cf* out, const cf* ahy, float scale,
                int subtract, cudaStream_t st) {
  const FPlan* fp = reinterpret_cast<const FPlan*>(c->fplan_raw);
  const int cpg = (c->Nc + G - 1) / G;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G, d.Ny, f);
  cfg.blockDim = dim3(kThreads, 1, 1);
  cfg.dynamicSmemBytes = smem_z(c, fp[2].npass);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = G;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const cf* T = c->d_T;
  const cf* smod = c->d_smaps_mod;
  if (c->zpre) {
    cfg.dynamicSmemBytes = smem_zadj_pre(c, fp[2].npass);
    MSLR_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_zadj_pre, T, smod, out, ahy, t0, scale, subtract, d,
                                     fp[2], (const cf*)c->d_tw[2], cpg));
  } else {
    MSLR_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_zadj_fast, T, smod, out, ahy, t0, scale, subtract, d,
                                     fp[2], (const cf*)c->d_tw[2], cpg));
  }
  return MSLR_OK;
}

}  // namespace

int normal_op_fast(Ctx* c, const cf* X, int ns, int64_t sstride, cf* g, bool subtract,
                   cudaStream_t st) {
  const Dims d = dims_of(c);
  const FPlan* fp = reinterpret_cast<const FPlan*>(c->fplan_raw);
  const float scale = (float)(1.0 / (double)c->nvox);
  const int G = groups_of(c->Nc);
  const int cpg = (c->Nc + G - 1) / G;
  for (int t0 = 0; t0 < c->Nt; t0 += c->Ffast) {
    const int f = std::min(c->Ffast, c->Nt - t0);
    if (c->zpre)
      k_zfwd_pre<<<dim3(G, d.Ny, f), kThreads, smem_zfwd_pre(c, fp[2].npass), st>>>(
          X, ns, sstride, t0, c->d_smaps_mod, c->d_T, d, fp[2], c->d_tw[2], cpg);
    else
      k_zfwd_fast<<<dim3(G, d.Ny, f), kThreads, smem_z(c, fp[2].npass), st>>>(
          X, ns, sstride, t0, c->d_smaps_mod, c->d_T, d, fp[2], c->d_tw[2], cpg);
    if (c->xypers) {
      const int units = d.Nz * d.Nc * f;
      k_xy_pers<<<std::min(units, c->nsm), kThreads, smem_xy_pers(c), st>>>(
          c->d_T, c->d_mask, c->nwords, t0, f, d, fp[0], fp[1], c->d_tw[0], c->d_tw[1]);
    } else {
      k_xy_fast<<<dim3(d.Nz, d.Nc, f), kThreads, smem_xy(c), st>>>(
          c->d_T, c->d_mask, c->nwords, t0, d, fp[0], fp[1], c->d_tw[0], c->d_tw[1], XY_NORMAL);
    }
    int rc = launch_zadj(c, d, G, f, t0, g, c->d_ahy, scale, subtract ? 1 : 0, st);
    if (rc) return rc;
    c->launches += 3;
  }
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int sense_forward_fast(Ctx* c, const cf* x, cf* y, cudaStream_t st) {
  const Dims d = dims_of(c);
  const FPlan* fp = reinterpret_cast<const FPlan*>(c->fplan_raw);
  const float s = (float)(1.0 / std::sqrt((double)c->nvox));
  const int G = groups_of(c->Nc);
  const int cpg = (c->Nc + G - 1) / G;
  for (int t0 = 0; t0 < c->Nt; t0 += c->Ffast) {
    const int f = std::min(c->Ffast, c->Nt - t0);
    k_zfwd_fast<<<dim3(G, d.Ny, f), kThreads, smem_z(c, fp[2].npass), st>>>(
        x, 1, 0, t0, c->d_smaps_mod, c->d_T, d, fp[2], c->d_tw[2], cpg);
    k_xy_fast<<<dim3(d.Nz, d.Nc, f), kThreads, smem_xy(c), st>>>(
        c->d_T, c->d_mask, c->nwords, t0, d, fp[0], fp[1], c->d_tw[0], c->d_tw[1], XY_FORWARD);
    const int gx = (int)std::min<int64_t>((c->K + 255) / 256, 64);
    k_gather_fast<<<dim3(gx, d.Nc, f), 256, 0, st>>>(c->d_T, c->d_idx, y, t0, c->K, s,
                                                      c->d_phase[0], c->d_phase[1],
                                                      c->d_phase[2], d);
    c->launches += 3;
  }
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int sense_adjoint_fast(Ctx* c, const cf* y, cf* x, cudaStream_t st) {
  const Dims d = dims_of(c);
  const FPlan* fp = reinterpret_cast<const FPlan*>(c->fplan_raw);
  const float s = (float)(1.0 / std::sqrt((double)c->nvox));
  const int G = groups_of(c->Nc);
  for (int t0 = 0; t0 < c->Nt; t0 += c->Ffast) {
    const int f = std::min(c->Ffast, c->Nt - t0);
    MSLR_CUDA_TRY(cudaMemsetAsync(c->d_T, 0, (size_t)f * d.Nc * d.nvox * sizeof(cf), st));
    const int gx = (int)std::min<int64_t>((c->K + 255) / 256, 64);
    k_scatter_fast<<<dim3(gx, d.Nc, f), 256, 0, st>>>(c->d_T, c->d_idx, y, t0, c->K, s,
                                                       c->d_phase[0], c->d_phase[1],
                                                       c->d_phase[2], d);
    k_xy_fast<<<dim3(d.Nz, d.Nc, f), kThreads, smem_xy(c), st>>>(
        c->d_T, c->d_mask, c->nwords, t0, d, fp[0], fp[1], c->d_tw[0], c->d_tw[1], XY_ADJOINT);
    int rc = launch_zadj(c, d, G, f, t0, x, nullptr, 1.0f, 0, st);
    if (rc) return rc;
    c->launches += 3;
  }
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

}  // namespace mslr
