// sense.cu — SENSE operator, adjoint and normal operator on sm_100a.
//
// Reference behaviour: src/sense_gpu.jl:56-108 (Asense_gpu, per frame:
// y = s·fftshift(fft(ifftshift(S_c x)))[idx], s = 1/sqrt(prod(N))) with the
// exact unitary adjoint, assembled block-diagonally over frames
// (scripts/reconstruct.jl:142-147), and the data-consistency gradient
// A'(A Σ_k X_k − y) of scripts/reconstruct.jl:180-183.
//
// Centring without data movement: with c = n/2 (integer division) per axis,
//   fftshift(fft(ifftshift(x)))[k] = φ(k) · DFT(m ⊙ x)[k],
//   m(j) = exp(2πi j c / n),  φ(k) = exp(2πi c (k − c) / n),
// so the coil maps are pre-multiplied by m once at bind time, and φ only
// appears where k-space samples enter or leave (gather/scatter).  In the
// normal operator the mask sits between a forward and a backward DFT, φ
// cancels (|φ| = 1), and A'A x = s² Σ_c conj(S'_c) bDFT(M_t ⊙ DFT(S'_c x)).
//
// Decomposition per frame (z-first, x fastest in memory):
//   k_zfwd : per (y, frame): Σ_k X_k → × S'_c → DFT along z, for every coil
//   k_xy   : per (kz, coil, frame) plane: DFT x, DFT y, mask, bDFT y, bDFT x
//   k_zadj : per (y, frame): bDFT along z → × conj(S'_c) → Σ_c, − A'y
// The per-coil k-space of a chunk of frames lives in ctx->d_T.
#include <cmath>
#include <cstdio>

#include "fft.cuh"
#include "internal.h"

namespace mslr {

namespace {

struct Dims {
  int Nx, Ny, Nz, Nc;
  int64_t nvox;
};

enum XyMode { XY_NORMAL = 0, XY_FORWARD = 1, XY_ADJOINT = 2 };

__device__ __forceinline__ void load_tw(cf* dst, const cf* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// ---------------------------------------------------------------------------
// bind-time kernels
// ---------------------------------------------------------------------------
__global__ void k_modmaps(const cf* __restrict__ smaps, cf* __restrict__ smod, const cf* mx,
                          const cf* my, const cf* mz, Dims d) {
  const int64_t total = (int64_t)d.Nc * d.nvox;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = i % d.nvox;
    const int x = (int)(v % d.Nx);
    const int y = (int)((v / d.Nx) % d.Ny);
    const int z = (int)(v / ((int64_t)d.Nx * d.Ny));
    smod[i] = cmul(smaps[i], cmul(mx[x], cmul(my[y], mz[z])));
  }
}

// Validate and rebase indices: in range and strictly ascending per frame
// (the reference's findall(vec(samp)) output).  err bit0: out of range,
// bit1: not strictly ascending.
__global__ void k_check_idx(const int32_t* __restrict__ in, int32_t* __restrict__ out, int base,
                            int Nt, int64_t K, int64_t nvox, int32_t* err) {
  const int64_t total = (int64_t)Nt * K;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = i % K;
    const int64_t k = (int64_t)in[i] - base;
    int bad = 0;
    if (k < 0 || k >= nvox) bad |= 1;
    if (j > 0 && in[i] <= in[i - 1]) bad |= 2;
    if (bad) atomicOr(err, bad);
    out[i] = (k < 0 || k >= nvox) ? 0 : (int32_t)k;
  }
}

__global__ void k_build_mask(const int32_t* __restrict__ idx, uint32_t* __restrict__ mask,
                             int Nt, int64_t K, int nwords) {
  const int64_t total = (int64_t)Nt * K;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(i / K);
    const int k = idx[i];
    atomicOr(&mask[(int64_t)t * nwords + (k >> 5)], 1u << (k & 31));
  }
}

// ---------------------------------------------------------------------------
// z pass, forward: per (y, frame).  xs[z][x] = Σ_k X_k[t][z][y][x]; for each
// coil, w = xs ⊙ S'_c, DFT along z, store to T[f][c][kz][y][x].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_zfwd(const cf* __restrict__ X, int ns, int64_t sstride,
                                              int t0, const cf* __restrict__ smod,
                                              cf* __restrict__ T, Dims d, AxisPlan pz,
                                              const cf* __restrict__ twz) {
  extern __shared__ cf sm[];
  const int S = d.Nz * d.Nx;
  cf* tw = sm;
  cf* xs = tw + d.Nz;
  cf* a = xs + S;
  cf* b = a + S;
  const int y = blockIdx.x;
  const int f = blockIdx.y;
  const int t = t0 + f;
  load_tw(tw, twz, d.Nz);
  const int64_t plane = (int64_t)d.Nx * d.Ny;
  for (int i = threadIdx.x; i < S; i += blockDim.x) {
    const int z = i / d.Nx, x = i - z * d.Nx;
    const int64_t off = (int64_t)t * d.nvox + z * plane + (int64_t)y * d.Nx + x;
    cf v = X[off];
    for (int k = 1; k < ns; ++k) v = cadd(v, X[off + k * sstride]);
    xs[i] = v;
  }
  __syncthreads();
  for (int c = 0; c < d.Nc; ++c) {
    const cf* sc = smod + (int64_t)c * d.nvox;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
      const int z = i / d.Nx, x = i - z * d.Nx;
      a[i] = cmul(xs[i], sc[z * plane + (int64_t)y * d.Nx + x]);
    }
    __syncthreads();
    cf* r = fft_lines<false>(a, b, pz, tw, d.Nx, d.Nx, 1);
    cf* Tc = T + ((int64_t)f * d.Nc + c) * d.nvox;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
      const int z = i / d.Nx, x = i - z * d.Nx;
      Tc[z * plane + (int64_t)y * d.Nx + x] = r[i];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// xy pass: per (kz, coil, frame) plane of T.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_xy(cf* __restrict__ T, const uint32_t* __restrict__ mask,
                                            int nwords, int t0, Dims d, AxisPlan px, AxisPlan py,
                                            const cf* __restrict__ twx_g,
                                            const cf* __restrict__ twy_g, int mode) {
  extern __shared__ cf sm[];
  const int P = d.Nx * d.Ny;
  cf* twx = sm;
  cf* twy = twx + d.Nx;
  cf* a = twy + d.Ny;
  cf* b = a + P;
  const int kz = blockIdx.x, c = blockIdx.y, f = blockIdx.z;
  const int t = t0 + f;
  load_tw(twx, twx_g, d.Nx);
  load_tw(twy, twy_g, d.Ny);
  cf* pl = T + ((int64_t)f * d.Nc + c) * d.nvox + (int64_t)kz * P;
  for (int i = threadIdx.x; i < P; i += blockDim.x) a[i] = pl[i];
  __syncthreads();
  cf* r = a;
  if (mode != XY_ADJOINT) {
    cf* o = (r == a) ? b : a;
    r = fft_lines<false>(r, o, px, twx, d.Ny, 1, d.Nx);   // along x (rows)
    o = (r == a) ? b : a;
    r = fft_lines<false>(r, o, py, twy, d.Nx, d.Nx, 1);   // along y (columns)
  }
  if (mode == XY_NORMAL) {
    const uint32_t* mk = mask + (int64_t)t * nwords;
    const int64_t base = (int64_t)kz * P;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
      const int64_t k = base + i;
      if (!((mk[k >> 5] >> (k & 31)) & 1u)) r[i] = make_float2(0.f, 0.f);
    }
    __syncthreads();
  }
  if (mode != XY_FORWARD) {
    cf* o = (r == a) ? b : a;
    r = fft_lines<true>(r, o, py, twy, d.Nx, d.Nx, 1);
    o = (r == a) ? b : a;
    r = fft_lines<true>(r, o, px, twx, d.Ny, 1, d.Nx);
  }
  for (int i = threadIdx.x; i < P; i += blockDim.x) pl[i] = r[i];
}

// ---------------------------------------------------------------------------
// z pass, adjoint: per (y, frame).  acc = Σ_c conj(S'_c) ⊙ bDFT_z(T_c);
// out = scale·acc − (subtract ? A'y : 0).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_zadj(const cf* __restrict__ T, const cf* __restrict__ smod,
                                              cf* __restrict__ out, const cf* __restrict__ ahy,
                                              int t0, float scale, int subtract, Dims d,
                                              AxisPlan pz, const cf* __restrict__ twz) {
  extern __shared__ cf sm[];
  const int S = d.Nz * d.Nx;
  cf* tw = sm;
  cf* acc = tw + d.Nz;
  cf* a = acc + S;
  cf* b = a + S;
  const int y = blockIdx.x;
  const int f = blockIdx.y;
  const int t = t0 + f;
  load_tw(tw, twz, d.Nz);
  const int64_t plane = (int64_t)d.Nx * d.Ny;
  for (int i = threadIdx.x; i < S; i += blockDim.x) acc[i] = make_float2(0.f, 0.f);
  for (int c = 0; c < d.Nc; ++c) {
    const cf* Tc = T + ((int64_t)f * d.Nc + c) * d.nvox;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
      const int z = i / d.Nx, x = i - z * d.Nx;
      a[i] = Tc[z * plane + (int64_t)y * d.Nx + x];
    }
    __syncthreads();
    cf* r = fft_lines<true>(a, b, pz, tw, d.Nx, d.Nx, 1);
    const cf* sc = smod + (int64_t)c * d.nvox;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
      const int z = i / d.Nx, x = i - z * d.Nx;
      acc[i] = cadd(acc[i], cmulc(sc[z * plane + (int64_t)y * d.Nx + x], r[i]));
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < S; i += blockDim.x) {
    const int z = i / d.Nx, x = i - z * d.Nx;
    const int64_t off = (int64_t)t * d.nvox + z * plane + (int64_t)y * d.Nx + x;
    cf v = cscale(acc[i], scale);
    if (subtract) v = csub(v, ahy[off]);
    out[off] = v;
  }
}

__device__ __forceinline__ cf phase_at(int64_t k, const cf* px, const cf* py, const cf* pz,
                                       const Dims& d) {
  const int x = (int)(k % d.Nx);
  const int y = (int)((k / d.Nx) % d.Ny);
  const int z = (int)(k / ((int64_t)d.Nx * d.Ny));
  return cmul(px[x], cmul(py[y], pz[z]));
}

// y[t][c][i] = s·φ(idx)·T[f][c][idx]
__global__ void k_gather(const cf* __restrict__ T, const int32_t* __restrict__ idx,
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

// T[f][c][idx] = s·conj(φ(idx))·y[t][c][i]   (T zeroed beforehand)
__global__ void k_scatter(cf* __restrict__ T, const int32_t* __restrict__ idx,
                          const cf* __restrict__ yin, int t0, int64_t K, float s, const cf* px,
                          const cf* py, const cf* pz, Dims d) {
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

size_t smem_z(const Ctx* c) { return sizeof(cf) * (c->N[2] + 3 * (size_t)c->N[2] * c->N[0]); }
size_t smem_xy(const Ctx* c) {
  return sizeof(cf) * (c->N[0] + c->N[1] + 2 * (size_t)c->N[0] * c->N[1]);
}

int make_plan(int n, AxisPlan* p) {
  p->n = n;
  p->npass = 0;
  int m = n;
  const int pref[] = {4, 5, 3, 2};
  while (m > 1) {
    int r = 0;
    for (int q : pref)
      if (m % q == 0) {
        r = q;
        break;
      }
    if (!r) {
      for (int q = 7; q <= kMaxRadix; ++q)
        if (m % q == 0) {
          r = q;
          break;
        }
    }
    if (!r || p->npass >= kMaxPasses) return 0;
    p->radix[p->npass++] = r;
    m /= r;
  }
  return 1;
}

}  // namespace

int sense_setup_tables(Ctx* c) {
  for (int ax = 0; ax < 3; ++ax) {
    const int n = c->N[ax];
    if (n < 1 || n > kMaxFftLen || !make_plan(n, &c->plan[ax]))
      return fail(MSLR_ERR_UNSUPPORTED,
                  "FFT axis length " + std::to_string(n) +
                      " unsupported (needs 1..1024 with prime factors <= 16)");
    std::vector<cf> tw(n), ph(n), md(n);
    const int cc = n / 2;
    for (int k = 0; k < n; ++k) {
      const double a = -2.0 * M_PI * (double)k / n;
      tw[k] = make_float2((float)std::cos(a), (float)std::sin(a));
      const double b = 2.0 * M_PI * (double)cc * (double)(k - cc) / n;
      ph[k] = make_float2((float)std::cos(b), (float)std::sin(b));
      const double e = 2.0 * M_PI * std::fmod((double)k * cc, (double)n) / n;
      md[k] = make_float2((float)std::cos(e), (float)std::sin(e));
    }
    int rc;
    if ((rc = dalloc(c, (void**)&c->d_tw[ax], n * sizeof(cf)))) return rc;
    if ((rc = dalloc(c, (void**)&c->d_phase[ax], n * sizeof(cf)))) return rc;
    if ((rc = dalloc(c, (void**)&c->d_mod[ax], n * sizeof(cf)))) return rc;
    MSLR_CUDA_TRY(cudaMemcpy(c->d_tw[ax], tw.data(), n * sizeof(cf), cudaMemcpyHostToDevice));
    MSLR_CUDA_TRY(cudaMemcpy(c->d_phase[ax], ph.data(), n * sizeof(cf), cudaMemcpyHostToDevice));
    MSLR_CUDA_TRY(cudaMemcpy(c->d_mod[ax], md.data(), n * sizeof(cf), cudaMemcpyHostToDevice));
  }
  const size_t sz = smem_z(c), sxy = smem_xy(c);
  if (sz > 227 * 1024 || sxy > 227 * 1024)
    return fail(MSLR_ERR_UNSUPPORTED, "image dimensions too large for the shared-memory FFT");
  MSLR_CUDA_TRY(raise_dyn_smem((const void*)k_zfwd, (int)sz));
  MSLR_CUDA_TRY(raise_dyn_smem((const void*)k_zadj, (int)sz));
  MSLR_CUDA_TRY(raise_dyn_smem((const void*)k_xy, (int)sxy));
  // frames per chunk: keep the per-coil k-space of a chunk near 0.6 GB
  const double per_frame = (double)c->Nc * c->nvox * sizeof(cf);
  int F = (int)std::max(1.0, std::floor(600e6 / per_frame));
  c->F = std::min(F, c->Nt);
  int rc = dalloc(c, (void**)&c->d_T, (size_t)c->F * c->Nc * c->nvox * sizeof(cf));
  if (rc) return rc;
  c->nwords = (int)((c->nvox + 31) / 32);
  // tuned form: register-resident kernels when every axis has a fast plan;
  // one frame per chunk so that the chunk's per-coil k-space can stay in L2
  if (c->tuned()) {
    c->fast = sense_fast_setup(c);
    c->spec = c->fast && sense_spec_setup(c);
  }
  c->Ffast = 1;
  return MSLR_OK;
}

int sense_bind(Ctx* c, const cf* smaps, const cf* y, const int32_t* idx, int base,
               cudaStream_t st) {
  int rc;
  const Dims d = dims_of(c);
  if (!c->d_smaps_mod) {
    if ((rc = dalloc(c, (void**)&c->d_smaps_mod, (size_t)c->Nc * c->nvox * sizeof(cf)))) return rc;
    if ((rc = dalloc(c, (void**)&c->d_mask, (size_t)c->Nt * c->nwords * sizeof(uint32_t)))) return rc;
    if ((rc = dalloc(c, (void**)&c->d_idx, (size_t)c->Nt * c->K * sizeof(int32_t)))) return rc;
    if ((rc = dalloc(c, (void**)&c->d_ahy, (size_t)c->Nt * c->nvox * sizeof(cf)))) return rc;
  }
  MSLR_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int32_t), st));
  k_check_idx<<<1184, 256, 0, st>>>(idx, c->d_idx, base, c->Nt, c->K, c->nvox, c->d_err);
  MSLR_CUDA_TRY(cudaGetLastError());
  int32_t herr = 0;
  MSLR_CUDA_TRY(cudaMemcpyAsync(&herr, c->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr & 1) return fail(MSLR_ERR_ARG, "sample index out of range for the image grid");
  if (herr & 2) return fail(MSLR_ERR_ARG, "sample indices must be strictly ascending per frame");
  MSLR_CUDA_TRY(cudaMemsetAsync(c->d_mask, 0, (size_t)c->Nt * c->nwords * sizeof(uint32_t), st));
  k_build_mask<<<1184, 256, 0, st>>>(c->d_idx, c->d_mask, c->Nt, c->K, c->nwords);
  k_modmaps<<<1184, 256, 0, st>>>(smaps, c->d_smaps_mod, c->d_mod[0], c->d_mod[1], c->d_mod[2], d);
  MSLR_CUDA_TRY(cudaGetLastError());
  c->bound = true;
  rc = sense_adjoint(c, y, c->d_ahy, st);
  if (!rc) rc = data_norm2(c, y, &c->ynorm2, st);   // ‖y‖² for dc_cost (cost.cu)
  if (rc) {
    c->bound = false;
    return rc;
  }
  return MSLR_OK;
}

int sense_forward(Ctx* c, const cf* x, cf* y, cudaStream_t st) {
  if (c->fast) return sense_forward_fast(c, x, y, st);
  const Dims d = dims_of(c);
  const float s = (float)(1.0 / std::sqrt((double)c->nvox));
  for (int t0 = 0; t0 < c->Nt; t0 += c->F) {
    const int f = std::min(c->F, c->Nt - t0);
    k_zfwd<<<dim3(d.Ny, f), 256, smem_z(c), st>>>(x, 1, 0, t0, c->d_smaps_mod, c->d_T, d,
                                                  c->plan[2], c->d_tw[2]);
    k_xy<<<dim3(d.Nz, d.Nc, f), 256, smem_xy(c), st>>>(c->d_T, c->d_mask, c->nwords, t0, d,
                                                       c->plan[0], c->plan[1], c->d_tw[0],
                                                       c->d_tw[1], XY_FORWARD);
    const int gx = (int)std::min<int64_t>((c->K + 255) / 256, 64);
    k_gather<<<dim3(gx, d.Nc, f), 256, 0, st>>>(c->d_T, c->d_idx, y, t0, c->K, s,
                                                 c->d_phase[0], c->d_phase[1], c->d_phase[2], d);
    c->launches += 3;
  }
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int sense_adjoint(Ctx* c, const cf* y, cf* x, cudaStream_t st) {
  if (c->fast) return sense_adjoint_fast(c, y, x, st);
  const Dims d = dims_of(c);
  const float s = (float)(1.0 / std::sqrt((double)c->nvox));
  for (int t0 = 0; t0 < c->Nt; t0 += c->F) {
    const int f = std::min(c->F, c->Nt - t0);
    MSLR_CUDA_TRY(cudaMemsetAsync(c->d_T, 0, (size_t)f * d.Nc * d.nvox * sizeof(cf), st));
    const int gx = (int)std::min<int64_t>((c->K + 255) / 256, 64);
    k_scatter<<<dim3(gx, d.Nc, f), 256, 0, st>>>(c->d_T, c->d_idx, y, t0, c->K, s,
                                                  c->d_phase[0], c->d_phase[1], c->d_phase[2], d);
    k_xy<<<dim3(d.Nz, d.Nc, f), 256, smem_xy(c), st>>>(c->d_T, c->d_mask, c->nwords, t0, d,
                                                       c->plan[0], c->plan[1], c->d_tw[0],
                                                       c->d_tw[1], XY_ADJOINT);
    k_zadj<<<dim3(d.Ny, f), 256, smem_z(c), st>>>(c->d_T, c->d_smaps_mod, x, nullptr, t0, 1.0f,
                                                  0, d, c->plan[2], c->d_tw[2]);
    c->launches += 3;
  }
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

int normal_op(Ctx* c, const cf* X, int ns, int64_t sstride, cf* g, bool subtract,
              cudaStream_t st) {
  if (c->spec) return normal_op_spec(c, X, ns, sstride, g, subtract, st);
  if (c->fast) return normal_op_fast(c, X, ns, sstride, g, subtract, st);
  const Dims d = dims_of(c);
  const float scale = (float)(1.0 / (double)c->nvox);
  for (int t0 = 0; t0 < c->Nt; t0 += c->F) {
    const int f = std::min(c->F, c->Nt - t0);
    k_zfwd<<<dim3(d.Ny, f), 256, smem_z(c), st>>>(X, ns, sstride, t0, c->d_smaps_mod, c->d_T, d,
                                                  c->plan[2], c->d_tw[2]);
    k_xy<<<dim3(d.Nz, d.Nc, f), 256, smem_xy(c), st>>>(c->d_T, c->d_mask, c->nwords, t0, d,
                                                       c->plan[0], c->plan[1], c->d_tw[0],
                                                       c->d_tw[1], XY_NORMAL);
    k_zadj<<<dim3(d.Ny, f), 256, smem_z(c), st>>>(c->d_T, c->d_smaps_mod, g, c->d_ahy, t0, scale,
                                                  subtract ? 1 : 0, d, c->plan[2], c->d_tw[2]);
    c->launches += 3;
  }
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

}  // namespace mslr
