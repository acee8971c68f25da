"""Seeded synthetic MSLR problems with the reference's shapes.

The reference reconstructs measured EPI k-space (``ksp_epi_zf``) with BART
coil maps; neither is available, so problems are generated from a seed.  The
generator follows the reference pipeline of scripts/reconstruct.jl:86-147:

1. coil maps are SOS-normalised as at scripts/reconstruct.jl:89,
2. the per-frame mask has the same sample count in every frame
   (asserted by the reference at scripts/reconstruct.jl:116-118),
3. k-space is divided by the 99th percentile of the SENSE-combined
   zero-filled image (scripts/reconstruct.jl:102-104, src/recon.jl:312-323).

Random draws use one ``numpy.random.Generator(PCG64(seed))`` in a fixed
order: spatial maps, temporal basis, image noise, coil-map parameters,
per-frame masks, k-space noise.

Layouts are the reference's column-major arrays read as C-order numpy arrays
with reversed axes: image (Nt, Nz, Ny, Nx), coil maps (Nc, Nz, Ny, Nx),
k-space (Nt, Nc, K), sample indices (Nt, K) 0-based ascending.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft

AX = (-3, -2, -1)


@dataclass
class SynthConfig:
    """Shape and distribution of one synthetic problem."""
    N: tuple = (32, 32, 24)
    Nc: int = 8
    Nt: int = 64
    rank: int = 4
    frac: float = 0.25
    centre: int = 8
    noise_x: float = 0.01
    noise_y: float = 0.01
    decay: float | None = None
    normalize: bool = True
    seed: int = 1234
    patch_sizes: list = field(default_factory=lambda: [[6, 6, 6]])
    strides: list = field(default_factory=lambda: [[6, 6, 6]])
    niters: int = 20


# Named workloads (sizes from the reference's experiment files and the
# benchmark definition): small CPU case, the 90x90x60 two-scale metric case,
# the three-scale half-overlapping case, and the differentiation case.
CONFIGS = {
    "small": SynthConfig(),
    "metric": SynthConfig(N=(90, 90, 60), Nc=18, Nt=300, rank=8, frac=1 / 6, centre=12,
                          patch_sizes=[[90, 90, 60], [10, 10, 10]],
                          strides=[[90, 90, 60], [10, 10, 10]], niters=50),
    "batching": SynthConfig(N=(90, 90, 60), Nc=18, Nt=387, rank=8, frac=1 / 6, centre=12,
                            patch_sizes=[[90, 90, 60], [10, 10, 10], [6, 6, 6]],
                            strides=[[90, 90, 60], [5, 5, 5], [3, 3, 3]], niters=50),
    "precision": SynthConfig(N=(90, 90, 60), Nc=18, Nt=300, rank=8, frac=1 / 6, centre=12,
                             decay=1.5, patch_sizes=[[90, 90, 60], [10, 10, 10]],
                             strides=[[90, 90, 60], [10, 10, 10]], niters=50),
    # the metric's image, coil and scale shapes with 8 frames: per-frame
    # kernels are identical, so this is the case profiled with ncu
    "profile": SynthConfig(N=(90, 90, 60), Nc=18, Nt=8, rank=8, frac=1 / 6, centre=12,
                           patch_sizes=[[90, 90, 60], [10, 10, 10]],
                           strides=[[90, 90, 60], [10, 10, 10]], niters=5),
    "diff": SynthConfig(N=(48, 48, 32), Nc=12, Nt=128, rank=8, frac=1 / 6, centre=8,
                        patch_sizes=[[48, 48, 32], [8, 8, 8]],
                        strides=[[48, 48, 32], [8, 8, 8]], niters=10),
}


def _cnormal(rng, shape, dtype=np.complex64):
    re = rng.standard_normal(shape, dtype=np.float32)
    im = rng.standard_normal(shape, dtype=np.float32)
    out = np.empty(shape, dtype=dtype)
    out.real = re
    out.imag = im
    out *= np.float32(1 / math.sqrt(2))
    return out


def coil_maps(rng, N, Nc):
    """Smooth Gaussian bumps centred on a sphere around the FOV, each with a
    smooth linear phase, SOS-normalised as scripts/reconstruct.jl:89."""
    Nx, Ny, Nz = N
    zs = np.linspace(-1, 1, Nz, dtype=np.float64)[:, None, None]
    ys = np.linspace(-1, 1, Ny, dtype=np.float64)[None, :, None]
    xs = np.linspace(-1, 1, Nx, dtype=np.float64)[None, None, :]
    golden = math.pi * (3 - math.sqrt(5))
    params = rng.standard_normal((Nc, 4))
    maps = np.empty((Nc, Nz, Ny, Nx), dtype=np.complex64)
    for c in range(Nc):
        zc = 1 - 2 * (c + 0.5) / Nc
        rc = math.sqrt(max(0.0, 1 - zc * zc))
        th = golden * c
        cx, cy, cz = 1.3 * rc * math.cos(th), 1.3 * rc * math.sin(th), 1.3 * zc
        d2 = (xs - cx) ** 2 + (ys - cy) ** 2 + (zs - cz) ** 2
        mag = np.exp(-d2 / (2 * 0.8 ** 2))
        ph = 0.5 * (params[c, 0] * xs + params[c, 1] * ys + params[c, 2] * zs) + math.pi * params[c, 3]
        maps[c] = (mag * np.exp(1j * ph)).astype(np.complex64)
    sos = np.sqrt(np.sum(np.abs(maps) ** 2, axis=0)).astype(np.float32)
    maps /= (sos + np.finfo(np.float32).eps)[None]
    return maps


def masks(rng, N, Nt, frac, centre):
    """Per-frame sample indices: a fully sampled centre cube plus uniformly
    random points, with the same count K in every frame.  Returns (Nt, K)
    int32, 0-based column-major linear indices, ascending per frame."""
    Nx, Ny, Nz = N
    nvox = Nx * Ny * Nz
    c = [min(centre, n) for n in N]
    lo = [n // 2 - cc // 2 for n, cc in zip(N, c)]
    zz, yy, xx = np.meshgrid(np.arange(lo[2], lo[2] + c[2]), np.arange(lo[1], lo[1] + c[1]),
                             np.arange(lo[0], lo[0] + c[0]), indexing="ij")
    centre_idx = np.sort((xx + Nx * (yy + Ny * zz)).ravel())
    K = max(int(round(frac * nvox)), centre_idx.size)
    is_centre = np.zeros(nvox, dtype=bool)
    is_centre[centre_idx] = True
    outside = np.flatnonzero(~is_centre)
    nrand = K - centre_idx.size
    idx = np.empty((Nt, K), dtype=np.int32)
    for t in range(Nt):
        pick = outside[rng.choice(outside.size, size=nrand, replace=False)]
        idx[t] = np.sort(np.concatenate([centre_idx, pick]))
    return idx


def sense_forward_c64(x, smaps, idx, workers=-1):
    """Centred unitary SENSE forward per frame in complex64 (generator use)."""
    Nt = x.shape[0]
    Nc = smaps.shape[0]
    K = idx.shape[1]
    nvox = x[0].size
    s = np.float32(1 / math.sqrt(nvox))
    y = np.empty((Nt, Nc, K), dtype=np.complex64)
    for t in range(Nt):
        kc = sfft.fftshift(sfft.fftn(sfft.ifftshift(smaps * x[t][None], axes=AX), axes=AX,
                                     workers=workers), axes=AX)
        y[t] = kc.reshape(Nc, -1)[:, idx[t]] * s
    return y


def _torch_forward(x, smaps, idx):
    """The same centred unitary forward with torch.fft on the GPU (input
    generation only; used for the full-size workloads)."""
    import torch
    dev = torch.device("cuda")
    S = torch.from_numpy(smaps).to(dev)
    Nt, Nc, K = x.shape[0], smaps.shape[0], idx.shape[1]
    s = 1.0 / math.sqrt(x[0].size)
    y = np.empty((Nt, Nc, K), dtype=np.complex64)
    for t in range(Nt):
        xt = torch.from_numpy(x[t]).to(dev)
        kc = torch.fft.fftshift(torch.fft.fftn(torch.fft.ifftshift(S * xt[None], dim=AX), dim=AX), dim=AX)
        it = torch.from_numpy(idx[t].astype(np.int64)).to(dev)
        y[t] = (kc.reshape(Nc, -1)[:, it] * s).cpu().numpy()
    return y


def _torch_comb_scale(y, smaps, idx, q=0.99):
    import torch
    dev = torch.device("cuda")
    S = torch.from_numpy(smaps).to(dev)
    Nt, Nc, K = y.shape
    _, Nz, Ny, Nx = smaps.shape
    nvox = Nx * Ny * Nz
    denom = (S.abs() ** 2).sum(0).double() + np.finfo(np.float64).eps
    mags = torch.empty((Nt, nvox), dtype=torch.float32, device=dev)
    for t in range(Nt):
        full = torch.zeros((Nc, nvox), dtype=torch.complex64, device=dev)
        full[:, torch.from_numpy(idx[t].astype(np.int64)).to(dev)] = torch.from_numpy(y[t]).to(dev)
        img = torch.fft.fftshift(torch.fft.ifftn(torch.fft.ifftshift(full.reshape(Nc, Nz, Ny, Nx), dim=AX),
                                                 dim=AX), dim=AX)
        num = (S.conj() * img).sum(0)
        mags[t] = (num.abs().double() / denom).float().reshape(-1)
    v = mags.reshape(-1)
    # numpy-style linear-interpolated quantile via two order statistics
    n = v.numel()
    pos = q * (n - 1)
    lo = int(math.floor(pos))
    vals = torch.sort(v).values
    a, b = float(vals[lo]), float(vals[min(lo + 1, n - 1)])
    return a + (b - a) * (pos - lo)


def sense_comb_scale(y, smaps, idx, q=0.99, workers=-1):
    """scale_factor = quantile(|sense_comb(ksp)|, 0.99) for the zero-filled
    k-space grid holding y (src/recon.jl:312-323, scripts/reconstruct.jl:102-103)."""
    Nt, Nc, K = y.shape
    _, Nz, Ny, Nx = smaps.shape
    nvox = Nx * Ny * Nz
    denom = np.sum(np.abs(smaps) ** 2, axis=0) + np.finfo(np.float64).eps
    mags = np.empty((Nt, Nz, Ny, Nx), dtype=np.float32)
    for t in range(Nt):
        full = np.zeros((Nc, nvox), dtype=np.complex64)
        full[:, idx[t]] = y[t]
        img_mc = sfft.fftshift(sfft.ifftn(sfft.ifftshift(full.reshape(Nc, Nz, Ny, Nx), axes=AX),
                                          axes=AX, workers=workers), axes=AX)
        num = np.sum(np.conj(smaps) * img_mc, axis=0)
        mags[t] = np.abs(num / denom)
    return float(np.quantile(mags.ravel(), q))


def make_problem(cfg: SynthConfig, workers: int = -1, fft: str = "scipy") -> dict:
    """Generate one problem.  Returns a dict with ``smaps``, ``idx``, ``y``,
    ``x_true`` (normalised by the same scale factor as y) and metadata.
    ``fft="torch"`` computes the k-space and the normalisation with
    torch.fft on the GPU (same random draws; used for full-size inputs)."""
    rng = np.random.Generator(np.random.PCG64(cfg.seed))
    Nx, Ny, Nz = cfg.N
    nvox = Nx * Ny * Nz
    r = cfg.rank
    M = _cnormal(rng, (nvox, r))
    if cfg.decay is not None:
        M *= (np.arange(1, r + 1, dtype=np.float32) ** np.float32(-cfg.decay))[None]
    B0 = _cnormal(rng, (cfg.Nt, r), dtype=np.complex128)
    B, _ = np.linalg.qr(B0)
    B = B.astype(np.complex64)
    x = (np.conj(B) @ M.T).reshape(cfg.Nt, Nz, Ny, Nx)          # x[t, v] = Σ_r M[v,r] conj(B[t,r])
    rms = float(np.sqrt(np.mean(np.abs(x) ** 2)))
    x += _cnormal(rng, x.shape) * np.float32(cfg.noise_x * rms)
    smaps = coil_maps(rng, cfg.N, cfg.Nc)
    idx = masks(rng, cfg.N, cfg.Nt, cfg.frac, cfg.centre)
    y = _torch_forward(x, smaps, idx) if fft == "torch" else sense_forward_c64(x, smaps, idx, workers)
    y += _cnormal(rng, y.shape) * np.float32(cfg.noise_y)
    scale = 1.0
    if cfg.normalize:
        sc = _torch_comb_scale(y, smaps, idx) if fft == "torch" else sense_comb_scale(y, smaps, idx,
                                                                                        workers=workers)
        scale = max(sc, float(np.finfo(np.float32).eps))
        y /= np.float32(scale)
        x /= np.float32(scale)
    return {"smaps": smaps, "idx": idx, "y": y, "x_true": x, "scale_factor": scale,
            "N": tuple(cfg.N), "Nc": cfg.Nc, "Nt": cfg.Nt, "K": idx.shape[1],
            "patch_sizes": [list(p) for p in cfg.patch_sizes],
            "strides": [list(s) for s in cfg.strides], "niters": cfg.niters}
