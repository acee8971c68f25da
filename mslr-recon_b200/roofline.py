"""Roofline denominators and algorithmic byte / flop counts per step.

Peaks come from MEASURED_PEAKS.json at the repository root (a STREAM-style
copy for HBM, cuBLAS bf16 for the tensor pipe); without it the fallback
figures measured earlier on the same GPU type are used.
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
