// patchmap.cuh — device-side addressing of patch elements (src/recon.jl:53-78
// geometry), shared by the SIMT and tensor-core patch kernels.
#pragma once
#include "common.cuh"

namespace mslr {

// Device-side addressing of patch elements.  Element (l, t) of patch ip —
// l the in-patch voxel (x fastest), t the frame — lives at
//   image mode: origin(ip) + lx + Nx (ly + Ny lz) + t·nvox
//   batch mode: ip·mstride + l + t·m        (column-major m × Nt matrices)
struct PatchMap {
  int Nx, Ny, Nz;
  int64_t nvox;
  int Nt;
  int psx, psy, psz;
  int nx, ny, nz;     // patches per dim
  const int* starts;  // nx x-starts, ny y-starts, nz z-starts
  int p, n, L;
  int tall;
  int batch;
  int64_t mstride;
};

__device__ __forceinline__ int64_t patch_origin(const PatchMap& m, int64_t ip) {
  if (m.batch) return ip * m.mstride;
  const int ix = (int)(ip % m.nx);
  const int iy = (int)((ip / m.nx) % m.ny);
  const int iz = (int)(ip / ((int64_t)m.nx * m.ny));
  const int sx = m.starts[ix], sy = m.starts[m.nx + iy], sz = m.starts[m.nx + m.ny + iz];
  return sx + (int64_t)m.Nx * (sy + (int64_t)m.Ny * sz);
}

__device__ __forceinline__ int64_t patch_off(const PatchMap& m, int l) {
  if (m.batch) return l;
  const int lx = l % m.psx;
  const int r = l / m.psx;
  const int ly = r % m.psy;
  const int lz = r / m.psy;
  return lx + (int64_t)m.Nx * (ly + (int64_t)m.Ny * lz);
}

__device__ __forceinline__ int64_t tstride(const PatchMap& m) { return m.batch ? (int64_t)m.p : m.nvox; }

// M[a][l] of patch with origin `org`
__device__ __forceinline__ cf m_elem(const PatchMap& m, const cf* __restrict__ img, int64_t org,
                                     int a, int l) {
  if (m.tall) {
    const cf v = img[org + patch_off(m, l) + (int64_t)a * tstride(m)];
    return cconj(v);
  }
  return img[org + patch_off(m, a) + (int64_t)l * tstride(m)];
}


// gram_umma.cu: split-precision BF16 (or TF32) patch Grams and rebuilds on
// tcgen05 for the tuned and TF32 forms.
// umma_supported: the 32-bit offset tables of those kernels cover this map.
bool umma_supported(const PatchMap& m);
int gram_umma_launch(const cf* img, const PatchMap& m, int64_t np, cf* out_or_part, int nsplit,
                     int lchunk, const DevWait& dw, cudaStream_t st, bool tf32 = false);
int rebuild_umma_launch(const cf* img, const cf* W, const PatchMap& m, int64_t np, cf* out,
                        int direct, const DevWait& dw, cudaStream_t st, bool tf32 = false);
int umma_prepare();

}  // namespace mslr
