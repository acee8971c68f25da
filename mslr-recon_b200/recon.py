"""Patch operators and SVST — the call surface of src/recon.jl and
src/sense_gpu.jl (img2patches, patches2img, SVST, patchSVST), backed by
libmslr kernels on CUDA tensors.

Layouts: an image time series is a C-order (Nt, Nz, Ny, Nx) complex64 tensor
(the memory of the reference's column-major (Nx, Ny, Nz, Nt) array); a patch
stack is (Np, Nt, p) (the reference's (p, Nt, Np)).  Patch sizes and strides
are (x, y, z) triples as in the reference.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import FORM_TUNED, check, i32arr, lib
from .context import _stream_ptr


def patch_geometry(N, patch_size, stride_size):
    """src/recon.jl:54-72.  Returns (ps, nsteps, Np, starts) with ps clamped
    to N, nsteps = cld(N - ps, ss) and 0-based starts per dimension."""
    ps = (C.c_int32 * 3)()
    ns = (C.c_int32 * 3)()
    Np = C.c_int64()
    check(lib.mslr_patch_geometry(i32arr(N), i32arr(patch_size), i32arr(stride_size), ps, ns,
                                  C.byref(Np), None))
    total = sum(int(v) + 1 for v in ns)
    st = (C.c_int32 * total)()
    check(lib.mslr_patch_geometry(i32arr(N), i32arr(patch_size), i32arr(stride_size), ps, ns,
                                  C.byref(Np), st))
    out, off = [], 0
    for d in range(3):
        c = int(ns[d]) + 1
        out.append([int(v) for v in st[off:off + c]])
        off += c
    return [int(v) for v in ps], [int(v) for v in ns], int(Np.value), out


def _img_dims(img):
    if img.dim() != 4 or img.dtype != torch.complex64 or not img.is_cuda:
        raise ValueError("img must be a CUDA complex64 tensor (Nt, Nz, Ny, Nx)")
    Nt, Nz, Ny, Nx = img.shape
    return (Nx, Ny, Nz), Nt


def img2patches(img: torch.Tensor, patch_size, stride_size, stream=None) -> torch.Tensor:
    """src/recon.jl:53-78 — (Nt,Nz,Ny,Nx) -> (Np, Nt, p)."""
    N, Nt = _img_dims(img)
    ps, _, Np, _ = patch_geometry(N, patch_size, stride_size)
    p = ps[0] * ps[1] * ps[2]
    P = torch.empty((Np, Nt, p), dtype=torch.complex64, device=img.device)
    check(lib.mslr_img2patches(i32arr(N), Nt, i32arr(patch_size), i32arr(stride_size),
                               img.contiguous().data_ptr(), P.data_ptr(), _stream_ptr(stream)))
    return P


def patches2img(P: torch.Tensor, patch_size, stride_size, og_size, stream=None) -> torch.Tensor:
    """src/recon.jl:96-126 — overlap average with clamped Float32 counts."""
    Np, Nt, p = P.shape
    Nx, Ny, Nz = (int(v) for v in og_size)
    img = torch.empty((Nt, Nz, Ny, Nx), dtype=torch.complex64, device=P.device)
    check(lib.mslr_patches2img(i32arr((Nx, Ny, Nz)), Nt, i32arr(patch_size), i32arr(stride_size),
                               P.contiguous().data_ptr(), img.data_ptr(), _stream_ptr(stream)))
    return img


def svst_batch(Xcm: torch.Tensor, m: int, n: int, betas, form: int = FORM_TUNED, stream=None):
    """SVST of `batch` column-major m × n matrices stored back to back in
    ``Xcm`` (flat or (batch, n, m) C-order).  Returns a tensor of the same
    shape."""
    batch = Xcm.numel() // (m * n)
    bet = (C.c_double * batch)(*[float(b) for b in betas])
    ws_bytes = C.c_size_t()
    check(lib.mslr_svst_batch_workspace(m, n, batch, C.byref(ws_bytes)))
    ws = torch.empty(int(ws_bytes.value), dtype=torch.uint8, device=Xcm.device)
    out = torch.empty_like(Xcm)
    check(lib.mslr_svst_batch(m, n, batch, bet, Xcm.contiguous().data_ptr(), out.data_ptr(),
                              ws.data_ptr(), ws_bytes.value, form, _stream_ptr(stream)))
    return out


def SVST(X: torch.Tensor, beta: float, stream=None) -> torch.Tensor:
    """src/recon.jl:183-211 / src/sense_gpu.jl:122-128 on one (m × n) matrix:
    U diag(max(S - β, 0)) Vᴴ, zero for a zero matrix."""
    if X.dim() != 2:
        raise ValueError("SVST expects a 2-D matrix")
    m, n = X.shape
    cm = X.t().contiguous()              # column-major memory of X
    out = svst_batch(cm, m, n, [beta], stream=stream)
    return out.reshape(n, m).t()


def patchSVST(img: torch.Tensor, beta, patch_size, stride_size, stream=None) -> torch.Tensor:
    """src/recon.jl:251-268 / src/sense_gpu.jl:138-160: extract, SVST every
    patch (global β or one λ per patch), recombine."""
    N, Nt = _img_dims(img)
    P = img2patches(img, patch_size, stride_size, stream)
    Np, _, p = P.shape
    betas = list(beta) if hasattr(beta, "__len__") else [float(beta)] * Np
    if len(betas) != Np:
        raise ValueError(f"need {Np} per-patch thresholds, got {len(betas)}")
    P = svst_batch(P, p, Nt, betas, stream=stream)
    return patches2img(P, patch_size, stride_size, N, stream)
