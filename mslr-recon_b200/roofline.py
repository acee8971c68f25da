"""Roofline denominators and algorithmic byte / flop counts per step.

Peaks come from MEASURED_PEAKS.json at the repository root (a STREAM-style
copy for HBM, cuBLAS bf16 for the tensor pipe); without it the fallback
figures measured earlier on the same GPU type are used.  The FP32 SIMT peak is
measured by the library's own FMA probe (mslr_fp32_peak) when the bench runs.

Byte counts are algorithmic: every array a step must read or write, once.
Flop counts are nominal: 5 N log2 N per complex FFT of length N, 6 per
complex multiply, 8 per complex multiply-add of a GEMM.
"""
from __future__ import annotations

import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}
C64 = 8


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "bf16_tflops_sustained": float(d.get("bf16_tflops_sustained", d["bf16_tflops"])),
                "source": "measured"}
    except Exception:
        return dict(FALLBACK, source="fallback")


def normal_op_bytes(nvox: int, Nt: int, Nc: int, Ns: int) -> int:
    """A'(A Σ_k X_k) − A'y per iteration: read Ns scale images and A'y,
    write g, read the coil maps once and the per-frame sampling bitmasks."""
    img = nvox * Nt * C64
    return Ns * img + img + img + Nc * nvox * C64 + Nt * ((nvox + 31) // 32) * 4


def normal_op_flops(nvox: int, Nt: int, Nc: int) -> float:
    """Nominal 5 N log2 N per complex 3-D FFT, forward and backward, per
    coil and frame."""
    import math
    return 2.0 * Nc * Nt * 5.0 * nvox * math.log2(nvox)


def plane_pass_bytes(Nx: int, Ny: int, planes: int) -> int:
    """Plane kernel (x/y transforms, mask, inverse): every k-space plane of
    the chunk is read once and written once, plus its sampling bits."""
    pl = Nx * Ny
    return planes * (2 * pl * C64 + (pl + 31) // 32 * 4)


def plane_pass_flops(Nx: int, Ny: int, planes: int) -> float:
    """Nominal 5 N log2 N for the forward and the backward 2-D transform of
    each plane (N = Nx·Ny)."""
    import math
    pl = Nx * Ny
    return planes * 2 * 5.0 * pl * math.log2(pl)


def svst_bytes(nvox: int, Nt: int) -> int:
    """One scale's patch SVST: read the scale image, write it back."""
    return 2 * nvox * Nt * C64


def svst_flops(p: int, Nt: int, Np: int) -> float:
    """Gram (8 p n²) and rebuild (8 p n²) real flops per patch, n = min(p, Nt)."""
    n = min(p, Nt)
    L = max(p, Nt)
    return Np * 2 * 8.0 * L * n * n


def pogm_update_bytes(nvox: int, Nt: int, Ns: int) -> int:
    """Fused u/z update: read x, u (Ns each) and g; write u and z (Ns each)."""
    img = nvox * Nt * C64
    return 4 * Ns * img + img


def _fft_flops(n: int) -> float:
    import math
    return 5.0 * n * math.log2(n)


def four_pass_kernels(N, ch: int, f: int) -> dict:
    """Per-launch algorithmic bytes and flops of the four kernels of one chunk
    (ch coils × f frames) of the four-pass SENSE normal operator."""
    Nx, Ny, Nz = N
    pl = Nx * Ny
    nvox = pl * Nz
    img = nvox * C64
    planes = ch * f * Nz
    mask_bits = f * ((nvox + 31) // 32) * 4
    return {
        # Σ_k X_k planes of f frames, the group's coil maps, the chunk's k-space written
        "pfwd": {"bytes": f * img + ch * img + ch * f * img,
                 "flops": planes * (_fft_flops(pl) + 6.0 * pl)},
        # the chunk's k-space read and written, the frames' sampling bits
        "zmask": {"bytes": 2 * ch * f * img + mask_bits,
                  "flops": ch * f * Ny * Nx * 2 * _fft_flops(Nz)},
        # the chunk's k-space read and written, the group's coil maps read
        "padj": {"bytes": 2 * ch * f * img + ch * img,
                 "flops": planes * (_fft_flops(pl) + 6.0 * pl)},
        # the chunk's k-space read, g (or A'y) read, g written
        "csum": {"bytes": ch * f * img + 2 * f * img, "flops": ch * f * nvox * 2.0},
    }


def eig_flops(n: int, Np: int) -> float:
    """Eigen stage of one scale: Householder tridiagonalisation of the n × n
    Hermitian Gram (16/3 n³ real flops) and the back-transform of all n
    vectors (8 n³)."""
    return Np * (16.0 / 3.0 + 8.0) * n ** 3


def iteration_steps(N, Nt: int, Nc: int, scales) -> list:
    """The POGM iteration as a list of steps (name, bytes, flops, pipe) with
    pipe ∈ {"fp32", "tensor_split_bf16"}: the SENSE normal operator, the fused
    update, and per scale the patch Grams and rebuilds (split-BF16 tensor
    products, three BF16 MMAs per FP32-accurate product) and the eigen stage.
    ``scales``: list of (p, Np)."""
    Nx, Ny, Nz = N
    nvox = Nx * Ny * Nz
    Ns = len(scales)
    steps = [("normal_op", normal_op_bytes(nvox, Nt, Nc, Ns), normal_op_flops(nvox, Nt, Nc), "fp32"),
             ("pogm_update", pogm_update_bytes(nvox, Nt, Ns), 0.0, "fp32")]
    for k, (p, Np) in enumerate(scales):
        n = min(p, Nt)
        gram_w = svst_flops(p, Nt, Np) + Np * 8.0 * n ** 3   # Gram + rebuild, and W = Ṽ Ṽᴴ
        steps.append((f"svst_products_{k}", svst_bytes(nvox, Nt), gram_w, "tensor_split_bf16"))
        steps.append((f"eigen_{k}", 0, eig_flops(n, Np), "fp32"))
    return steps


def iteration_bound_seconds(steps, hbm_gbs: float, fp32_tflops: float, bf16_tflops: float) -> float:
    """Σ over steps of max(bytes / HBM bandwidth, flops / the step's peak)."""
    tot = 0.0
    for _, byts, fl, pipe in steps:
        peak = fp32_tflops if pipe == "fp32" else bf16_tflops / 3.0
        tot += max(byts / (hbm_gbs * 1e9), fl / (peak * 1e12) if fl else 0.0)
    return tot
