// svst.cu — batched patch SVST on sm_100a (plain FP32 SIMT form).
//
// Reference: img2patches / patches2img (src/recon.jl:53-126), SVST
// (src/recon.jl:183-211; src/sense_gpu.jl:122-128) and patchSVST
// (src/recon.jl:251-269; src/sense_gpu.jl:138-160).
//
// For a patch matrix P (p × Nt) let n = min(p, Nt) and M be the n × L matrix
//   M = Pᴴ (p ≥ Nt, "tall")   or   M = P (p < Nt, "wide"),
// so that G = M Mᴴ is the smaller Gram matrix.  With G = V diag(λ) Vᴴ and
// σ = √λ, SVST(P) = U diag(max(σ − β, 0)) Vᴴ equals
//   W = V diag(h) Vᴴ,  h = max(σ − β, 0)/σ,   M_out = W M,
// and P_out = M_outᴴ (tall) or M_out (wide).  Zero patches give G = 0, no
// eigenvalue above β², W = 0 and a zero output: the reference's zero-norm
// skip (src/recon.jl:185) falls out without a special case.
//
// Per patch (one CTA):
//   Gram (this file) → eigen stage producing W (eig.cu) → rebuild (this file).
// Patches never see a host loop: every stage is one launch over all patches
// of a scale.  Overlapping or gapped patch grids are recombined by a gather
// over covering patches in ascending ip order with the Float32 coverage
// count, clamped to 1 (src/recon.jl:113-124).
#include <algorithm>
#include <cmath>
#include <atomic>
#include <mutex>

#include <cstdlib>
#include <string>

#include "internal.h"
#include "patchmap.cuh"

namespace mslr {

// Poll count of the bounded waits in context-free calls (mslr_svst_batch,
// mslr_svst_batch_noalloc); contexts carry their own (Ctx::wait_polls).
static std::atomic<int> g_free_polls{kWaitPolls};
int context_free_polls() { return g_free_polls.load(); }
void set_context_free_polls(int polls) { g_free_polls.store(polls); }

namespace {

constexpr int kTile = 64;
constexpr int kKc = 16;

// ---------------------------------------------------------------------------
// Gram: G[a][b] = Σ_l M[a][l] conj(M[b][l]) on lower-triangle 64×64 tiles.
// grid (ntri, Np, nsplit).  Output column-major: G[b*n + a].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_gram(const cf* __restrict__ img, PatchMap m,
                                              cf* __restrict__ out, int nsplit, int lchunk) {
  __shared__ cf As[kKc][kTile + 1];
  __shared__ cf Bs[kKc][kTile + 1];
  // tile pair from the linear lower-triangle index
  int t = blockIdx.x, ta = 0;
  while (t > ta) {
    t -= ta + 1;
    ++ta;
  }
  const int tb = t;
  const int64_t ip = blockIdx.y;
  const int split = blockIdx.z;
  const int64_t org = patch_origin(m, ip);
  const int a0 = ta * kTile, b0 = tb * kTile;
  const int l_begin = split * lchunk;
  const int l_end = min(m.L, l_begin + lchunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  cf acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
  for (int l0 = l_begin; l0 < l_end; l0 += kKc) {
    // load: 1024 elements each for A and B; kk fastest for tall (voxel-contiguous)
    for (int q = threadIdx.x; q < kKc * kTile; q += blockDim.x) {
      int kk, r;
      if (m.tall) {
        kk = q % kKc;
        r = q / kKc;
      } else {
        r = q % kTile;
        kk = q / kTile;
      }
      const int l = l0 + kk;
      cf va = make_float2(0.f, 0.f), vb = make_float2(0.f, 0.f);
      if (l < l_end) {
        if (a0 + r < m.n) va = m_elem(m, img, org, a0 + r, l);
        if (b0 + r < m.n) vb = m_elem(m, img, org, b0 + r, l);
      }
      As[kk][r] = va;
      Bs[kk][r] = vb;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kKc; ++kk) {
      cf av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          // av * conj(bv)
          acc[i][j].x += av[i].x * bv[j].x + av[i].y * bv[j].y;
          acc[i][j].y += av[i].y * bv[j].x - av[i].x * bv[j].y;
        }
    }
    __syncthreads();
  }
  const int n = m.n;
  cf* G = out + ((nsplit > 1) ? (int64_t)split * n * n : ip * (int64_t)n * n);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int a = a0 + ty * 4 + i, b = b0 + tx * 4 + j;
      if (a < n && b < n) {
        G[(int64_t)b * n + a] = acc[i][j];
        if (ta != tb) G[(int64_t)a * n + b] = cconj(acc[i][j]);
      }
    }
}

__global__ void k_gram_reduce(const cf* __restrict__ part, cf* __restrict__ G, int nsplit,
                              int64_t nn) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nn;
       e += (int64_t)gridDim.x * blockDim.x) {
    cf s = part[e];
    for (int q = 1; q < nsplit; ++q) s = cadd(s, part[q * nn + e]);
    G[e] = s;
  }
}

// ---------------------------------------------------------------------------
// Rebuild: M_out = W M.  tall: out[t=a][vox_l] = Σ_b conj(W[a][b]) img[b][vox_l]
//                       wide: out[t=l][vox_a] = Σ_b W[a][b] img[l][vox_b]
// grid (ceil(n/64), ceil(L/64), Np).  Writes the image directly when the
// patch grid is an exact partition, else the per-patch buffer (p, Nt, Np).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_rebuild(const cf* __restrict__ img, const cf* __restrict__ W,
                                                 PatchMap m, cf* __restrict__ out, int direct) {
  __shared__ cf As[kKc][kTile + 1];   // W[a][b]
  __shared__ cf Bs[kKc][kTile + 1];   // input values for (b, l)
  const int a0 = blockIdx.x * kTile, l0 = blockIdx.y * kTile;
  const int64_t ip = blockIdx.z;
  const int n = m.n;
  const cf* Wp = W + ip * (int64_t)n * n;
  const int64_t org = patch_origin(m, ip);
  const int64_t ts = tstride(m);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  cf acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
  for (int b0 = 0; b0 < n; b0 += kKc) {
    for (int q = threadIdx.x; q < kKc * kTile; q += blockDim.x) {
      // W tile: a fastest (column-major W[b*n + a])
      {
        const int r = q % kTile, kk = q / kTile;
        const int a = a0 + r, b = b0 + kk;
        cf w = make_float2(0.f, 0.f);
        if (a < n && b < n) {
          w = Wp[(int64_t)b * n + a];
          if (m.tall) w = cconj(w);
        }
        As[kk][r] = w;
      }
      // input tile
      {
        int kk, r;
        if (m.tall) {   // img[b][vox_l]: l contiguous
          r = q % kTile;
          kk = q / kTile;
        } else {        // img[l][vox_b]: b contiguous
          kk = q % kKc;
          r = q / kKc;
        }
        const int b = b0 + kk, l = l0 + r;
        cf v = make_float2(0.f, 0.f);
        if (b < n && l < m.L) {
          v = m.tall ? img[org + patch_off(m, l) + (int64_t)b * ts]
                     : img[org + patch_off(m, b) + (int64_t)l * ts];
        }
        Bs[kk][r] = v;
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kKc; ++kk) {
      cf av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x += av[i].x * bv[j].x - av[i].y * bv[j].y;
          acc[i][j].y += av[i].x * bv[j].y + av[i].y * bv[j].x;
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int a = a0 + ty * 4 + i, l = l0 + tx * 4 + j;
      if (a >= n || l >= m.L) continue;
      // element (voxel, frame) of the patch
      const int pv = m.tall ? l : a;
      const int tt = m.tall ? a : l;
      if (direct) out[org + patch_off(m, pv) + (int64_t)tt * ts] = acc[i][j];
      else out[(ip * m.Nt + tt) * (int64_t)m.p + pv] = acc[i][j];
    }
}

// img2patches: P[(ip*Nt + t)*p + l] = img[t][vox(ip, l)]
__global__ void k_img2patches(const cf* __restrict__ img, PatchMap m, cf* __restrict__ P,
                              int64_t total) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int l = (int)(q % m.p);
    const int64_t r = q / m.p;
    const int t = (int)(r % m.Nt);
    const int64_t ip = r / m.Nt;
    P[q] = img[patch_origin(m, ip) + patch_off(m, l) + (int64_t)t * m.nvox];
  }
}

// Gather recombine (patches2img): for voxel v and frame t, Σ over covering
// patches in ascending ip of P[(ip*Nt + t)*p + l(v, ip)], divided by
// max(count, 1).  cover: per dim 2*N[d] ints (lo, hi) of covering indices.
__global__ void k_recombine(const cf* __restrict__ P, PatchMap m, const int* __restrict__ cover,
                            cf* __restrict__ img) {
  const int64_t total = (int64_t)m.Nt * m.nvox;
  const int* cx = cover;
  const int* cy = cover + 2 * m.Nx;
  const int* cz = cy + 2 * m.Ny;
  const int* sxs = m.starts;
  const int* sys = m.starts + m.nx;
  const int* szs = m.starts + m.nx + m.ny;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = q % m.nvox;
    const int t = (int)(q / m.nvox);
    const int x = (int)(v % m.Nx);
    const int y = (int)((v / m.Nx) % m.Ny);
    const int z = (int)(v / ((int64_t)m.Nx * m.Ny));
    const int xl = cx[2 * x], xh = cx[2 * x + 1];
    const int yl = cy[2 * y], yh = cy[2 * y + 1];
    const int zl = cz[2 * z], zh = cz[2 * z + 1];
    cf acc = make_float2(0.f, 0.f);
    float cnt = 0.f;
    if (xl >= 0 && yl >= 0 && zl >= 0) {
      for (int iz = zl; iz <= zh; ++iz)
        for (int iy = yl; iy <= yh; ++iy)
          for (int ix = xl; ix <= xh; ++ix) {
            const int64_t ip = ix + (int64_t)m.nx * (iy + (int64_t)m.ny * iz);
            const int l = (x - sxs[ix]) + m.psx * ((y - sys[iy]) + m.psy * (z - szs[iz]));
            acc = cadd(acc, P[(ip * m.Nt + t) * (int64_t)m.p + l]);
            cnt += 1.f;
          }
    }
    cnt = fmaxf(cnt, 1.f);
    img[q] = make_float2(acc.x / cnt, acc.y / cnt);
  }
}

__global__ void k_zero(cf* p, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    p[q] = make_float2(0.f, 0.f);
}

PatchMap map_of(const ScaleGeom& g, const int N[3], int Nt, int64_t nvox) {
  PatchMap m;
  m.Nx = N[0];
  m.Ny = N[1];
  m.Nz = N[2];
  m.nvox = nvox;
  m.Nt = Nt;
  m.psx = g.ps[0];
  m.psy = g.ps[1];
  m.psz = g.ps[2];
  m.nx = g.nsteps[0] + 1;
  m.ny = g.nsteps[1] + 1;
  m.nz = g.nsteps[2] + 1;
  m.starts = g.d_starts;
  m.p = g.p;
  m.n = g.n;
  m.L = g.L;
  m.tall = g.tall ? 1 : 0;
  m.batch = 0;
  m.mstride = 0;
  return m;
}


struct WorkPtrs {
  cf* gram;
  void* zv;
  double* aux;
  double* vecs;
  int* rank;
  cf* part;
};

// Gram matrices of all patches described by m into w.gram.
// Tensor cores (tc, tuned form: split-precision BF16 mma) or FP32 SIMT.
int svst_gram(const cf* in, const PatchMap& m, int64_t np, const WorkPtrs& w, int nsplit, int tc,
              const DevWait& dw, cudaStream_t st, uint64_t* launches) {
  if (launches) *launches += (nsplit > 1 ? 2 : 1);
  const int n = m.n;
  const int T = (n + kTile - 1) / kTile;
  const int ntri = T * (T + 1) / 2;
  const int lchunk = (nsplit > 1) ? ((m.L + nsplit - 1) / nsplit + 31) / 32 * 32 : m.L;
  cf* dst = (nsplit > 1) ? w.part : w.gram;
  if (tc && umma_supported(m)) {
    if (int rc = gram_umma_launch(in, m, np, dst, nsplit, lchunk, dw, st, tc == 2)) return rc;
  } else {
    k_gram<<<dim3(ntri, (unsigned)np, nsplit), 256, 0, st>>>(in, m, dst, nsplit, lchunk);
  }
  if (nsplit > 1) k_gram_reduce<<<592, 256, 0, st>>>(w.part, w.gram, nsplit, (int64_t)n * n);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

// out (image when direct, else per-patch buffer) = rebuild with W in w.gram.
int svst_rebuild(const cf* in, const PatchMap& m, int64_t np, const WorkPtrs& w, cf* out,
                 int direct, int tc, const DevWait& dw, cudaStream_t st, uint64_t* launches) {
  if (launches) *launches += 1;
  if (tc && umma_supported(m))
    return rebuild_umma_launch(in, w.gram, m, np, out, direct, dw, st, tc == 2);
  const int n = m.n;
  k_rebuild<<<dim3((n + kTile - 1) / kTile, (m.L + kTile - 1) / kTile, (unsigned)np), 256, 0, st>>>(
      in, w.gram, m, out, direct);
  MSLR_CUDA_TRY(cudaGetLastError());
  return MSLR_OK;
}

// W = Ṽ Ṽᴴ for every patch, from the eigen stage's Ṽ (stored conjugated,
// row-major, in w.zv) into w.gram: the Gram of n × n matrices read as "tall"
// batch patches, M[a][l] = conj(zv[a·n + l]) = Ṽ[a][l].
int svst_form_w(const WorkPtrs& w, int n, int64_t np, int tc, const DevWait& dw, cudaStream_t st,
                uint64_t* launches) {
  PatchMap vm{};
  vm.batch = 1;
  vm.tall = 1;
  vm.Nt = n;
  vm.p = n;
  vm.n = n;
  vm.L = n;
  vm.nvox = n;
  vm.mstride = (int64_t)n * n;
  return svst_gram(reinterpret_cast<const cf*>(w.zv), vm, np, w, 1, tc, dw, st, launches);
}

// Gram → eig → W → (rebuild into out or pbuf) for all patches described by m.
int svst_core(const cf* in, const PatchMap& m, int64_t np, const WorkPtrs& w, int nsplit,
              const double* thr, int thr_per_patch, double lam, cf* out, int direct, int tc,
              const DevWait& dw, cudaStream_t st, uint64_t* launches, int eig_big = 0) {
  int rc = svst_gram(in, m, np, w, nsplit, tc, dw, st, launches);
  if (rc) return rc;
  rc = eig2_launch(m.n, np, w.gram, reinterpret_cast<cf*>(w.zv), reinterpret_cast<float*>(w.aux),
                   w.rank, thr, thr_per_patch, lam, st, eig_big, w.vecs, launches);
  if (rc) return rc;
  if ((rc = svst_form_w(w, m.n, np, tc, dw, st, launches))) return rc;
  return svst_rebuild(in, m, np, w, out, direct, tc, dw, st, launches);
}

// Split-K partial Grams are laid out one n × n block per split, so only a
// single-patch scale (the global patch) is split.
int choose_split(int64_t np, int n, int L) {
  if (np != 1) return 1;
  const int T = (n + kTile - 1) / kTile;
  const int64_t ctas = (int64_t)T * (T + 1) / 2 * np;
  if (ctas >= 592) return 1;
  int s = (int)std::min<int64_t>((592 + ctas - 1) / ctas, std::max(1, L / 1024));
  return std::max(1, s);
}

// the Gram's split-K count of a scale: the autotuner's choice when made
int split_of(const ScaleGeom& g) {
  return g.nsplit_tuned > 0 ? g.nsplit_tuned : choose_split(g.Np, g.n, g.L);
}

}  // namespace

// ---------------------------------------------------------------------------
// geometry (host)
// ---------------------------------------------------------------------------
int geom_build(const int N[3], int Nt, const int ps_in[3], const int ss_in[3], ScaleGeom* g) {
  int64_t Np = 1;
  g->h_starts.clear();
  bool partition = true;
  for (int d = 0; d < 3; ++d) {
    if (ps_in[d] <= 0 || ss_in[d] <= 0)
      return fail(MSLR_ERR_ARG, "patch sizes and strides must be positive");
    g->ps[d] = std::min(ps_in[d], N[d]);
    g->ss[d] = ss_in[d];
    const int num = N[d] - g->ps[d];
    g->nsteps[d] = (num + g->ss[d] - 1) / g->ss[d];   // cld for num >= 0
    Np *= (g->nsteps[d] + 1);
    int prev = -1;
    for (int i = 0; i <= g->nsteps[d]; ++i) {
      const int s = std::min(i * g->ss[d], N[d] - g->ps[d]);
      g->h_starts.push_back(s);
      if (i == 0 && s != 0) partition = false;
      if (i > 0 && s - prev != g->ps[d]) partition = false;
      prev = s;
    }
    if (prev + g->ps[d] != N[d]) partition = false;
  }
  g->Np = Np;
  g->p = g->ps[0] * g->ps[1] * g->ps[2];
  g->n = std::min(g->p, Nt);
  g->L = std::max(g->p, Nt);
  g->tall = g->p >= Nt;
  g->partition = partition;
  g->global = (Np == 1 && g->ps[0] == N[0] && g->ps[1] == N[1] && g->ps[2] == N[2]);
  g->d_starts = nullptr;
  g->d_cover = nullptr;
  return MSLR_OK;
}

int geom_upload(ScaleGeom* g, const int N[3]) {
  std::vector<int> cover;
  size_t off = 0;
  for (int d = 0; d < 3; ++d) {
    const int cnt = g->nsteps[d] + 1;
    for (int c = 0; c < N[d]; ++c) {
      int lo = -1, hi = -1;
      for (int i = 0; i < cnt; ++i) {
        const int s = g->h_starts[off + i];
        if (s <= c && c < s + g->ps[d]) {
          if (lo < 0) lo = i;
          hi = i;
        }
      }
      cover.push_back(lo);
      cover.push_back(hi);
    }
    off += cnt;
  }
  MSLR_CUDA_TRY(cudaMalloc((void**)&g->d_starts, g->h_starts.size() * sizeof(int)));
  MSLR_CUDA_TRY(cudaMemcpy(g->d_starts, g->h_starts.data(), g->h_starts.size() * sizeof(int),
                           cudaMemcpyHostToDevice));
  MSLR_CUDA_TRY(cudaMalloc((void**)&g->d_cover, cover.size() * sizeof(int)));
  MSLR_CUDA_TRY(cudaMemcpy(g->d_cover, cover.data(), cover.size() * sizeof(int),
                           cudaMemcpyHostToDevice));
  return MSLR_OK;
}

void geom_free(ScaleGeom* g) {
  if (g->d_starts) cudaFree(g->d_starts);
  if (g->d_cover) cudaFree(g->d_cover);
  g->d_starts = nullptr;
  g->d_cover = nullptr;
}

static size_t eig_work_bytes(int64_t np, int n, int nsplit) {
  const size_t nn = (size_t)n * n;
  return np * nn * sizeof(cf) * 2 + np * nn * sizeof(double) + np * 6 * (size_t)n * sizeof(double) +
         np * sizeof(int) + (nsplit > 1 ? (size_t)nsplit * nn * sizeof(cf) : 0) + 6 * 256;
}

static WorkPtrs carve(void* base, int64_t np, int n, int nsplit) {
  const size_t nn = (size_t)n * n;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  unsigned char* p = reinterpret_cast<unsigned char*>(base);
  WorkPtrs w;
  w.gram = reinterpret_cast<cf*>(p);
  p += al(np * nn * sizeof(cf));
  w.zv = p;
  p += al(np * nn * sizeof(cf));
  w.aux = reinterpret_cast<double*>(p);
  p += al(np * nn * sizeof(double));
  w.vecs = reinterpret_cast<double*>(p);
  p += al(np * 6 * (size_t)n * sizeof(double));
  w.rank = reinterpret_cast<int*>(p);
  p += al(np * sizeof(int));
  w.part = nsplit > 1 ? reinterpret_cast<cf*>(p) : nullptr;
  return w;
}

int svst_setup(Ctx* c) {
  size_t need = 0, pbuf = 0;
  for (auto& g : c->scales) {
    const int nsplit = choose_split(g.Np, g.n, g.L);
    need = std::max(need, eig_work_bytes(g.Np, g.n, nsplit));
    if (!g.partition) pbuf = std::max(pbuf, (size_t)g.Np * c->Nt * g.p);
  }
  int rc;
  // plain form: one workspace reused scale after scale; tuned form: one per
  // scale, so that every patch of every scale is in flight in one eigen launch
  const int nws = c->tuned() ? c->Ns : 1;
  c->svw.resize(nws);
  for (int k = 0; k < nws; ++k) {
    const ScaleGeom& g = c->scales[k];
    const size_t bytes = (nws == 1) ? need
                                    : eig_work_bytes(g.Np, g.n, choose_split(g.Np, g.n, g.L));
    void* base = nullptr;
    if ((rc = dalloc(c, &base, bytes))) return rc;
    c->svw[k].gram = reinterpret_cast<cf*>(base);
  }
  if (pbuf) {
    if ((rc = dalloc(c, (void**)&c->d_pbuf, pbuf * sizeof(cf)))) return rc;
    c->pbuf_elems = pbuf;
  }
  if ((rc = dalloc(c, (void**)&c->d_img_tmp, (size_t)c->Nt * c->nvox * sizeof(cf)))) return rc;
  {
    int64_t npmax = 1;
    for (auto& g : c->scales) npmax = std::max(npmax, g.Np);
    if ((rc = dalloc(c, (void**)&c->d_pthr, (size_t)npmax * sizeof(double)))) return rc;
  }
  int nmax = 1;
  for (auto& g : c->scales) nmax = std::max(nmax, g.n);
  if ((rc = umma_prepare())) return rc;   // before any graph capture of the iteration
  return eig2_prepare(nmax);
}

int patch_svst(Ctx* c, int s, const double* thr_dev, double lam, const cf* img_in, cf* img_out,
               cudaStream_t st, int thr_per_patch) {
  const ScaleGeom& g = c->scales[s];
  const PatchMap m = map_of(g, c->N, c->Nt, c->nvox);
  const int nsplit = split_of(g);
  WorkPtrs w = carve(c->svw[c->svw.size() > 1 ? s : 0].gram, g.Np, g.n, nsplit);
  const int tc = c->tc_mode();
  int rc;
  if (g.partition) {
    cf* dst = img_out;
    if (img_in == img_out) dst = c->d_img_tmp;   // Gram/rebuild read the input throughout
    if ((rc = svst_core(img_in, m, g.Np, w, nsplit, thr_dev, thr_per_patch, lam, dst, 1, tc, ctx_wait(c), st,
                        &c->launches, g.eig_big)))
      return rc;
    if (dst != img_out)
      MSLR_CUDA_TRY(cudaMemcpyAsync(img_out, dst, (size_t)c->Nt * c->nvox * sizeof(cf),
                                    cudaMemcpyDeviceToDevice, st));
  } else {
    if ((rc = svst_core(img_in, m, g.Np, w, nsplit, thr_dev, thr_per_patch, lam, c->d_pbuf, 0, tc,
                        ctx_wait(c), st, &c->launches, g.eig_big)))
      return rc;
    k_recombine<<<1184, 256, 0, st>>>(c->d_pbuf, m, g.d_cover, img_out);
    MSLR_CUDA_TRY(cudaGetLastError());
    c->launches += 1;
  }
  return MSLR_OK;
}

int patch_svst_lambdas(Ctx* c, int s, const double* lambdas_host, const cf* img_in, cf* img_out,
                       cudaStream_t st) {
  const ScaleGeom& g = c->scales[s];
  MSLR_CUDA_TRY(cudaMemcpyAsync(c->d_pthr, lambdas_host, (size_t)g.Np * sizeof(double), cudaMemcpyHostToDevice,
                                st));
  return patch_svst(c, s, c->d_pthr, 1.0, img_in, img_out, st, 1);
}

// Per-patch Σσ of scale s (patch_nucnorm's costs[ip], src/recon.jl:138-146):
// Grams of every patch, then the eigen stage in values-only mode.
int patch_nucnorms(Ctx* c, int k, const cf* X, std::vector<double>& h, cudaStream_t st) {
  const ScaleGeom& g = c->scales[k];
  int rc;
  if (c->nuc_cap < g.Np) {
    if (c->d_nuc) cudaFree(c->d_nuc);
    c->d_nuc = nullptr;
    c->nuc_cap = 0;
    int64_t npmax = 0;
    for (auto& gg : c->scales) npmax = std::max(npmax, gg.Np);
    if ((rc = dalloc(c, (void**)&c->d_nuc, (size_t)npmax * sizeof(double)))) return rc;
    c->nuc_cap = npmax;
  }
  if (!c->d_zero) {
    if ((rc = dalloc(c, (void**)&c->d_zero, sizeof(double)))) return rc;
    MSLR_CUDA_TRY(cudaMemsetAsync(c->d_zero, 0, sizeof(double), st));
  }
  const PatchMap m = map_of(g, c->N, c->Nt, c->nvox);
  const int nsplit = choose_split(g.Np, g.n, g.L);
  WorkPtrs w = carve(c->svw[c->svw.size() > 1 ? k : 0].gram, g.Np, g.n, nsplit);
  if ((rc = svst_gram(X, m, g.Np, w, nsplit, c->tc_mode(), ctx_wait(c), st, &c->launches))) return rc;
  EigSegment seg;
  seg.n = g.n;
  seg.np = g.Np;
  seg.gram = w.gram;
  seg.zv = reinterpret_cast<cf*>(w.zv);
  seg.aux = w.aux;
  seg.rank = w.rank;
  seg.lam = 0.0;
  seg.nuc = c->d_nuc;
  if ((rc = eig_launch_multi(1, &seg, c->d_zero, 0, st))) return rc;
  c->launches += 1;
  h.resize((size_t)g.Np);
  MSLR_CUDA_TRY(cudaMemcpyAsync(h.data(), c->d_nuc, (size_t)g.Np * sizeof(double), cudaMemcpyDeviceToHost, st));
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  return MSLR_OK;
}

// The Gram matrix (n × n, column-major) of the one patch of a single-patch
// scale s of img, into gram_out.  Sharded reconstructions add these partial
// Grams over the ranks' slabs of a tall global patch (G = Pᴴ P is a sum over
// voxels) and hand the sum to patch_svst_from_gram.
int patch_gram_out(Ctx* c, int s, const cf* img, cf* gram_out, cudaStream_t st) {
  const ScaleGeom& g = c->scales[s];
  if (g.Np != 1) return fail(MSLR_ERR_ARG, "the scale has more than one patch");
  const PatchMap m = map_of(g, c->N, c->Nt, c->nvox);
  const int nsplit = split_of(g);
  WorkPtrs w = carve(c->svw[c->svw.size() > 1 ? s : 0].gram, g.Np, g.n, nsplit);
  int rc;
  if ((rc = svst_gram(img, m, 1, w, nsplit, c->tc_mode(), ctx_wait(c), st, &c->launches))) return rc;
  MSLR_CUDA_TRY(cudaMemcpyAsync(gram_out, w.gram, (size_t)g.n * g.n * sizeof(cf), cudaMemcpyDeviceToDevice,
                                st));
  return MSLR_OK;
}

// SVST of the one patch of a single-patch scale s with threshold beta from a
// given Gram matrix (n × n, column-major): eigen stage, W, rebuild of
// img_in's patch into img_out (img_in may equal img_out).
int patch_svst_from_gram(Ctx* c, int s, double beta, const cf* gram, const cf* img_in, cf* img_out,
                         cudaStream_t st) {
  const ScaleGeom& g = c->scales[s];
  if (g.Np != 1) return fail(MSLR_ERR_ARG, "the scale has more than one patch");
  const PatchMap m = map_of(g, c->N, c->Nt, c->nvox);
  WorkPtrs w = carve(c->svw[c->svw.size() > 1 ? s : 0].gram, 1, g.n, split_of(g));
  const int tc = c->tc_mode();
  int rc;
  if ((rc = set_scalar(c->d_thr + 1, beta, st))) return rc;
  MSLR_CUDA_TRY(cudaMemcpyAsync(w.gram, gram, (size_t)g.n * g.n * sizeof(cf), cudaMemcpyDeviceToDevice, st));
  if ((rc = eig2_launch(g.n, 1, w.gram, reinterpret_cast<cf*>(w.zv), reinterpret_cast<float*>(w.aux), w.rank,
                        c->d_thr + 1, 0, 1.0, st, 0, w.vecs, &c->launches)))
    return rc;
  if ((rc = svst_form_w(w, g.n, 1, tc, ctx_wait(c), st, &c->launches))) return rc;
  cf* dst = g.partition ? img_out : c->d_pbuf;
  if (g.partition && img_in == img_out) dst = c->d_img_tmp;
  if ((rc = svst_rebuild(img_in, m, 1, w, dst, g.partition ? 1 : 0, tc, ctx_wait(c), st, &c->launches)))
    return rc;
  if (!g.partition) {
    k_recombine<<<1184, 256, 0, st>>>(c->d_pbuf, m, g.d_cover, img_out);
    MSLR_CUDA_TRY(cudaGetLastError());
    c->launches += 1;
  } else if (dst != img_out) {
    MSLR_CUDA_TRY(cudaMemcpyAsync(img_out, dst, (size_t)c->Nt * c->nvox * sizeof(cf), cudaMemcpyDeviceToDevice,
                                  st));
  }
  return MSLR_OK;
}

// g_prox of run_recon (scripts/reconstruct.jl:196-202) for every scale at once:
// Grams of all scales, one eigen launch per CTA variant over every patch of
// every scale (the global patch's eigensolve overlaps the local patches'),
// then the rebuilds.
// Zin / Xout are (Ns, Nt, Nz, Ny, Nx); threshold of scale k = (*thr_dev)·λ_k.
//
// When every scale's patches tile the volume exactly (no shared recombine
// buffer), the scales instead run as concurrent branches — each its own
// Gram → eigen → W → rebuild chain — forked from and joined back into st by
// events (legal inside a stream capture).  The scale with the fewest patches
// (the global patch) is issued first: its eigensolve takes a slot of the
// first wave, and its W Gram and rebuild then run on the SMs the larger
// scale's eigen launch leaves idle in its last wave.
int patch_svst_all(Ctx* c, const double* thr_dev, const cf* Zin, cf* Xout, cudaStream_t st) {
  const int64_t E = (int64_t)c->Nt * c->nvox;
  bool branches = c->Ns >= 2 && c->Ns <= 8 && c->svw.size() == (size_t)c->Ns;
  for (const auto& g : c->scales) branches = branches && g.partition;
  {
    const char* e = std::getenv("MSLR_SVST_BRANCHES");
    if (e && std::string(e) == "0") branches = false;
  }
  if (branches) {
    const int ns = c->Ns;
    if (c->sv_streams.size() < (size_t)ns - 1) {
      if (!c->sv_fork) MSLR_CUDA_TRY(cudaEventCreateWithFlags(&c->sv_fork, cudaEventDisableTiming));
      while (c->sv_streams.size() < (size_t)ns - 1) {
        cudaStream_t x;
        cudaEvent_t e;
        MSLR_CUDA_TRY(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
        MSLR_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->sv_streams.push_back(x);
        c->sv_join.push_back(e);
      }
    }
    std::vector<int> order(ns);
    for (int k = 0; k < ns; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return c->scales[a].Np < c->scales[b].Np; });
    MSLR_CUDA_TRY(cudaEventRecord(c->sv_fork, st));
    for (int i = 0; i + 1 < ns; ++i) MSLR_CUDA_TRY(cudaStreamWaitEvent(c->sv_streams[i], c->sv_fork, 0));
    int rc = MSLR_OK;
    for (int i = 0; i < ns && !rc; ++i) {   // side branches first, the largest scale on st
      const int k = order[i];
      cudaStream_t sk = (i + 1 < ns) ? c->sv_streams[i] : st;
      rc = patch_svst(c, k, thr_dev, c->lambdas[k], Zin + k * E, Xout + k * E, sk);
    }
    for (int i = 0; i + 1 < ns; ++i) {   // join every branch, also after an error
      cudaEventRecord(c->sv_join[i], c->sv_streams[i]);
      cudaStreamWaitEvent(st, c->sv_join[i], 0);
    }
    return rc;
  }
  if (c->svw.size() != (size_t)c->Ns) {
    for (int k = 0; k < c->Ns; ++k) {
      int rc = patch_svst(c, k, thr_dev, c->lambdas[k], Zin + k * E, Xout + k * E, st);
      if (rc) return rc;
    }
    return MSLR_OK;
  }
  std::vector<EigSegment> segs(c->Ns);
  std::vector<WorkPtrs> ws(c->Ns);
  int rc;
  for (int k = 0; k < c->Ns; ++k) {
    const ScaleGeom& g = c->scales[k];
    const PatchMap m = map_of(g, c->N, c->Nt, c->nvox);
    const int nsplit = split_of(g);
    ws[k] = carve(c->svw[k].gram, g.Np, g.n, nsplit);
    if ((rc = svst_gram(Zin + k * E, m, g.Np, ws[k], nsplit, c->tc_mode(), ctx_wait(c), st, &c->launches)))
      return rc;
    segs[k].n = g.n;
    segs[k].np = g.Np;
    segs[k].gram = ws[k].gram;
    segs[k].zv = reinterpret_cast<cf*>(ws[k].zv);
    segs[k].aux = ws[k].aux;
    segs[k].rank = ws[k].rank;
    segs[k].lam = c->lambdas[k];
    segs[k].big = g.eig_big;
    segs[k].side = ws[k].vecs;
  }
  if ((rc = eig_launch_multi(c->Ns, segs.data(), thr_dev, 0, st, &c->launches))) return rc;
  for (int k = 0; k < c->Ns; ++k)
    if ((rc = svst_form_w(ws[k], c->scales[k].n, c->scales[k].Np, c->tc_mode(), ctx_wait(c), st,
                          &c->launches)))
      return rc;
  for (int k = 0; k < c->Ns; ++k) {
    const ScaleGeom& g = c->scales[k];
    const PatchMap m = map_of(g, c->N, c->Nt, c->nvox);
    if (g.partition) {
      if ((rc = svst_rebuild(Zin + k * E, m, g.Np, ws[k], Xout + k * E, 1, c->tc_mode(), ctx_wait(c), st,
                             &c->launches)))
        return rc;
    } else {
      if ((rc = svst_rebuild(Zin + k * E, m, g.Np, ws[k], c->d_pbuf, 0, c->tc_mode(), ctx_wait(c), st,
                             &c->launches)))
        return rc;
      k_recombine<<<1184, 256, 0, st>>>(c->d_pbuf, m, g.d_cover, Xout + k * E);
      MSLR_CUDA_TRY(cudaGetLastError());
      c->launches += 1;
    }
  }
  return MSLR_OK;
}

// ---------------------------------------------------------------------------
// context-free entry points
// ---------------------------------------------------------------------------
int patches_op(const int N[3], int Nt, const int ps[3], const int ss[3], const cf* src, cf* dst,
               bool to_patches, cudaStream_t st) {
  ScaleGeom g;
  int rc = geom_build(N, Nt, ps, ss, &g);
  if (rc) return rc;
  if ((rc = geom_upload(&g, N))) {
    geom_free(&g);
    return rc;
  }
  const int64_t nvox = (int64_t)N[0] * N[1] * N[2];
  const PatchMap m = map_of(g, N, Nt, nvox);
  if (to_patches) {
    const int64_t total = g.Np * Nt * (int64_t)g.p;
    k_img2patches<<<1184, 256, 0, st>>>(src, m, dst, total);
  } else {
    k_recombine<<<1184, 256, 0, st>>>(src, m, g.d_cover, dst);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  geom_free(&g);
  if (e != cudaSuccess) return fail(MSLR_ERR_CUDA, cudaGetErrorString(e));
  return MSLR_OK;
}

// Workspace of the batched SVST: the eigen-stage work arrays, the thresholds,
// an error word and a staging copy of the input (for in == out).
size_t svst_batch_bytes(int mrows, int ncols, int batch) {
  const int n = std::min(mrows, ncols);
  return eig_work_bytes(batch, n, 1) + (size_t)batch * sizeof(double) + 256 + 256 +
         (size_t)batch * mrows * ncols * sizeof(cf) + 256;
}

// Runs every stage on st, then synchronises st and reads the call's error
// word: a bounded wait that ran out in a tensor-core kernel makes the call
// return MSLR_ERR_CUDA, and `out` is then not valid.
int svst_batch(int mrows, int ncols, int batch, const double* betas, const cf* in, cf* out,
               void* ws, size_t ws_bytes, int form, cudaStream_t st) {
  const int n = std::min(mrows, ncols);
  const size_t need = svst_batch_bytes(mrows, ncols, batch);
  if (ws_bytes < need) return fail(MSLR_ERR_ARG, "workspace too small for mslr_svst_batch");
  WorkPtrs w = carve(ws, batch, n, 1);
  unsigned char* tail = reinterpret_cast<unsigned char*>(ws) + eig_work_bytes(batch, n, 1);
  tail = reinterpret_cast<unsigned char*>(((uintptr_t)tail + 255) & ~(uintptr_t)255);
  double* d_beta = reinterpret_cast<double*>(tail);
  tail += ((size_t)batch * sizeof(double) + 255) & ~(size_t)255;
  int* d_err = reinterpret_cast<int*>(tail);
  tail += 256;
  cf* stage = reinterpret_cast<cf*>(tail);
  MSLR_CUDA_TRY(cudaMemcpyAsync(d_beta, betas, batch * sizeof(double), cudaMemcpyHostToDevice, st));
  MSLR_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), st));
  PatchMap m;
  m.Nx = mrows;
  m.Ny = 1;
  m.Nz = 1;
  m.nvox = mrows;
  m.Nt = ncols;
  m.psx = mrows;
  m.psy = 1;
  m.psz = 1;
  m.nx = m.ny = m.nz = 1;
  m.starts = nullptr;
  m.p = mrows;
  m.n = n;
  m.L = std::max(mrows, ncols);
  m.tall = mrows >= ncols;
  m.batch = 1;
  m.mstride = (int64_t)mrows * ncols;
  int rc = eig2_prepare(n);
  if (rc) return rc;
  const cf* src = in;
  if (in == out) {
    MSLR_CUDA_TRY(cudaMemcpyAsync(stage, in, (size_t)batch * mrows * ncols * sizeof(cf),
                                  cudaMemcpyDeviceToDevice, st));
    src = stage;
  }
  const int tc = form == MSLR_FORM_TF32 ? 2 : form == MSLR_FORM_TUNED ? 1 : 0;
  DevWait dw;
  dw.err = d_err;
  dw.polls = context_free_polls();
  if ((rc = svst_core(src, m, batch, w, 1, d_beta, 1, 1.0, out, 1, tc, dw, st, nullptr))) return rc;
  int herr = 0;
  MSLR_CUDA_TRY(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr & kErrMmaWait)
    return fail(MSLR_ERR_CUDA, "a tensor-core kernel's bounded wait for its MMAs timed out; "
                               "the output is not valid");
  return MSLR_OK;
}

// ---------------------------------------------------------------------------
// Batched SVST without any allocation, for callers that cannot call
// cudaMalloc (see mslr_svst_batch_noalloc in include/mslr.h).  Its scratch is
// this file-scope device array: every GPU that loads the library holds it
// until the process exits, and all calls share it.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[MSLR_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch, looked up once per device.  In host
// code the symbol name is only a host-side stand-in, so the kernels must be
// given the address that cudaGetSymbolAddress returns for the current device.
static void* g_noalloc_addr[64];
static std::mutex g_noalloc_mu;

int svst_batch_noalloc(int mrows, int ncols, int batch, const double* betas, const cf* in, cf* out,
                       cudaStream_t st) {
  const size_t need = svst_batch_bytes(mrows, ncols, batch);
  if (need > (size_t)MSLR_NOALLOC_SCRATCH_BYTES)
    return fail(MSLR_ERR_ARG,
                "mslr_svst_batch_noalloc: this batch needs " + std::to_string(need) +
                    " bytes of scratch, more than the fixed " +
                    std::to_string((size_t)MSLR_NOALLOC_SCRATCH_BYTES) +
                    " bytes; use mslr_svst_batch with a caller workspace or split the batch");
  int dev = 0;
  MSLR_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(MSLR_ERR_UNSUPPORTED, "device ordinal above 63");
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return fail(MSLR_ERR_CUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") +
                                       cudaGetErrorString(e));
      g_noalloc_addr[dev] = p;
    }
    scratch = g_noalloc_addr[dev];
  }
  // The array keeps the previous call's contents.  Only the error word has to
  // start at zero, and svst_batch clears it on the stream before the first
  // kernel; every other stage writes what the next one reads.
  return svst_batch(mrows, ncols, batch, betas, in, out, scratch, (size_t)MSLR_NOALLOC_SCRATCH_BYTES,
                    MSLR_FORM_TUNED, st);
}

// reg_cost of run_recon (scripts/reconstruct.jl:185-194): Σ_k λ_k Σ_patches
// Σ σ(P_p(X_k)) (patch_nucnorm, src/recon.jl:138-146).  The singular values of
// each patch are the square roots of its Gram's eigenvalues: Grams of every
// patch, then the eigen stage in values-only mode (tridiagonalisation and FP64
// bisection, no vectors).  Per-patch sums come back to the host and are added
// in patch order in FP64.  Synchronises st.
int patch_nucnorm_all(Ctx* c, const cf* X, double* reg_out, cudaStream_t st) {
  const int64_t E = (int64_t)c->Nt * c->nvox;
  std::vector<double> h;
  double reg = 0.0;
  for (int k = 0; k < c->Ns; ++k) {
    if (int rc = patch_nucnorms(c, k, X + k * E, h, st)) return rc;
    double sk = 0.0;
    for (double v : h) sk += v;
    reg += c->lambdas[k] * sk;
  }
  *reg_out = reg;
  return MSLR_OK;
}


// ---------------------------------------------------------------------------
// Patch-SVST backward (used by the unrolled-POGM gradient, grad.cu)
// ---------------------------------------------------------------------------
namespace {

struct VjpPtrs {
  cf* gram;     // np × n × n: G, then the Householder vectors
  cf* V;        // np × n × n: eigenvectors (row-major)
  double* aux;  // np × n × n: FP64 scratch of the eigen stage
  int* rank;    // np
  double* lam;  // np × n eigenvalues (descending)
  cf* wbar;     // W̄, then W
  cf* t1;       // W̄ V, then V diag(f), then V E
  cf* d;        // Vᴴ W̄ V, then K
  cf* e;        // F ⊙ (D + Dᴴ)
  double* bbar; // np
  cf* part;     // split-K partial products of the single-patch scale
};

int xsplit_of(int64_t np, int n, int L) {
  if (np != 1) return 1;
  const int T = (n + kTile - 1) / kTile;
  return std::max(1, std::min((592 + T * T - 1) / (T * T), std::max(1, L / 1024)));
}

size_t vjp_bytes(int64_t np, int n, int nsplit) {
  const size_t nn = (size_t)n * n;
  return np * nn * sizeof(cf) * 6 + np * nn * sizeof(double) + np * sizeof(int) +
         np * (size_t)n * sizeof(double) + np * sizeof(double) + (size_t)nsplit * nn * sizeof(cf) +
         11 * 256;
}

VjpPtrs carve_vjp(void* base, int64_t np, int n, int nsplit) {
  const size_t nn = (size_t)n * n;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  unsigned char* p = reinterpret_cast<unsigned char*>(base);
  auto take = [&](size_t bytes) {
    unsigned char* q = p;
    p += al(bytes);
    return q;
  };
  VjpPtrs v;
  v.gram = reinterpret_cast<cf*>(take(np * nn * sizeof(cf)));
  v.V = reinterpret_cast<cf*>(take(np * nn * sizeof(cf)));
  v.aux = reinterpret_cast<double*>(take(np * nn * sizeof(double)));
  v.rank = reinterpret_cast<int*>(take(np * sizeof(int)));
  v.lam = reinterpret_cast<double*>(take(np * (size_t)n * sizeof(double)));
  v.wbar = reinterpret_cast<cf*>(take(np * nn * sizeof(cf)));
  v.t1 = reinterpret_cast<cf*>(take(np * nn * sizeof(cf)));
  v.d = reinterpret_cast<cf*>(take(np * nn * sizeof(cf)));
  v.e = reinterpret_cast<cf*>(take(np * nn * sizeof(cf)));
  v.bbar = reinterpret_cast<double*>(take(np * sizeof(double)));
  v.part = reinterpret_cast<cf*>(take((size_t)nsplit * nn * sizeof(cf)));
  return v;
}

int nsplit_vjp(const ScaleGeom& g) {
  return std::max(choose_split(g.Np, g.n, g.L), xsplit_of(g.Np, g.n, g.L));
}

}  // namespace

int svst_vjp_setup(Ctx* c) {
  size_t need = 0;
  for (auto& g : c->scales) need = std::max(need, vjp_bytes(g.Np, g.n, nsplit_vjp(g)));
  if (need <= c->vjpw_bytes) return MSLR_OK;
  if (c->d_vjpw) cudaFree(c->d_vjpw);
  c->d_vjpw = nullptr;
  c->vjpw_bytes = 0;
  int rc;
  if ((rc = dalloc(c, &c->d_vjpw, need))) return rc;
  c->vjpw_bytes = need;
  return MSLR_OK;
}

// zbar = J_prox(z)ᴴ xbar for scale s (patch SVST with threshold β), and
// *bbar = ∂⟨xbar, prox(z)⟩/∂β.  tmp: one image of scratch.
int svst_vjp_scale(Ctx* c, int s, const cf* z, const cf* xbar, double beta, cf* zbar, cf* tmp,
                   double* bbar, cudaStream_t st) {
  const ScaleGeom& g = c->scales[s];
  const PatchMap m = map_of(g, c->N, c->Nt, c->nvox);
  const int64_t np = g.Np;
  const int n = g.n;
  const VjpPtrs v = carve_vjp(c->d_vjpw, np, n, nsplit_vjp(g));
  int rc;
  const cf* ob = xbar;
  if (!g.partition) {
    if ((rc = div_count_launch(xbar, m, g.d_cover, tmp, st))) return rc;
    ob = tmp;
  }
  WorkPtrs w{};
  w.gram = v.gram;
  w.zv = v.V;
  w.aux = v.aux;
  w.rank = v.rank;
  w.part = v.part;
  if ((rc = svst_gram(z, m, np, w, choose_split(np, n, g.L), 0, ctx_wait(c), st, &c->launches))) return rc;
  EigSegment seg;
  seg.n = n;
  seg.np = np;
  seg.gram = v.gram;
  seg.zv = v.V;
  seg.aux = v.aux;
  seg.rank = v.rank;
  seg.lam = 0.0;
  seg.lam_out = v.lam;
  if ((rc = eig_launch_multi(1, &seg, c->d_thr, 0, st))) return rc;
  if ((rc = xgram_launch(ob, z, m, np, v.wbar, v.part, xsplit_of(np, n, g.L), st))) return rc;
  if ((rc = bgemm_launch(0, 0, v.wbar, v.V, v.t1, n, np, st))) return rc;         // W̄ V
  if ((rc = bgemm_launch(1, 0, v.V, v.t1, v.d, n, np, st))) return rc;            // D = Vᴴ W̄ V
  if ((rc = divdiff_launch(v.d, v.lam, v.V, beta, n, np, v.e, v.t1, v.bbar, st))) return rc;
  if ((rc = bgemm_launch(0, 1, v.t1, v.V, v.wbar, n, np, st))) return rc;         // W = V f Vᴴ
  if ((rc = bgemm_launch(0, 0, v.V, v.e, v.t1, n, np, st))) return rc;            // V E
  if ((rc = bgemm_launch(0, 1, v.t1, v.V, v.d, n, np, st))) return rc;            // K = V E Vᴴ
  if (g.partition) {
    if ((rc = vjp_rebuild_launch(ob, z, v.wbar, v.d, m, np, zbar, 1, st))) return rc;
  } else {
    if ((rc = vjp_rebuild_launch(ob, z, v.wbar, v.d, m, np, c->d_pbuf, 0, st))) return rc;
    if ((rc = patch_sum_launch(c->d_pbuf, m, g.d_cover, zbar, st))) return rc;
  }
  c->launches += 11;
  std::vector<double> hb((size_t)np);
  MSLR_CUDA_TRY(cudaMemcpyAsync(hb.data(), v.bbar, np * sizeof(double), cudaMemcpyDeviceToHost, st));
  MSLR_CUDA_TRY(cudaStreamSynchronize(st));
  double t = 0.0;
  for (double x : hb) t += x;
  *bbar = t;
  return MSLR_OK;
}

// Autotuner: split-K count of the Gram of every single-patch scale (the
// global patch), among the counts its workspace holds, timed on A'y.
int tune_svst_splits(Ctx* c, cudaStream_t st) {
  for (size_t k = 0; k < c->scales.size(); ++k) {
    ScaleGeom& g = c->scales[k];
    if (g.Np != 1) continue;
    const int cap = choose_split(g.Np, g.n, g.L);
    const PatchMap m = map_of(g, c->N, c->Nt, c->nvox);
    float best = 1e30f;
    int bs = cap;
    for (int ns = cap; ns >= 1; ns = (ns > 1 && ns / 2 == 0) ? 1 : ns / 2) {
      WorkPtrs w = carve(c->svw[c->svw.size() > 1 ? k : 0].gram, g.Np, g.n, ns);
      float ms = 0.f;
      int rc = time_ms(st, 3, &ms, [&] {
        return svst_gram(c->d_ahy, m, 1, w, ns, c->tc_mode(), ctx_wait(c), st, nullptr);
      });
      if (rc) return rc;
      if (ms < best) {
        best = ms;
        bs = ns;
      }
      if (ns == 1) break;
    }
    g.nsplit_tuned = bs;
  }
  return MSLR_OK;
}

// Eigen-stage CTA variant of each scale whose Gram side allows both (n <= 384):
// 384 threads, two patches per SM, or 1024 threads, one per SM — timed on the
// scale's patch SVST of A'y at the threshold 1/Ns · λ_k (a first POGM
// iteration's ζ·λ_k with σ1 = 1), into the POGM z buffer (scratch until the
// first step).
int tune_eig_variants(Ctx* c, cudaStream_t st) {
  double* thr = c->d_thr + 3;
  if (int rc = set_scalar(thr, 1.0 / (double)c->Ns, st)) return rc;
  for (size_t k = 0; k < c->scales.size(); ++k) {
    ScaleGeom& g = c->scales[k];
    if (g.n > 384) {
      g.eig_big = 0;
      continue;
    }
    float best = 1e30f;
    int bb = 0;
    for (int big = 0; big <= 1; ++big) {
      g.eig_big = big;
      float ms = 0.f;
      int rc = time_ms(st, 2, &ms, [&] {
        return patch_svst(c, (int)k, thr, c->lambdas[k], c->d_ahy, c->d_Z, st, 0);
      });
      if (rc) return rc;
      if (ms < best) {
        best = ms;
        bb = big;
      }
    }
    g.eig_big = bb;
  }
  return MSLR_OK;
}

}  // namespace mslr
