"""run_recon on in-memory arrays — the hot part of scripts/reconstruct.jl:59-263.

File loading (scripts/reconstruct.jl:86-105) and saving (:241-262) are the
caller's business; this module takes coil maps, sampled k-space and sample
indices, builds the context, and runs POGM (mom=:pogm, restart=:gr) on the
device.  It returns what run_recon saves, minus the files.
"""
from __future__ import annotations

import numpy as np
import torch

from .context import MSLRContext


def sos_normalize(smaps: np.ndarray) -> np.ndarray:
    """scripts/reconstruct.jl:89: S ./ (sqrt(Σ_c |S_c|²) .+ eps(Float32))."""
    sos = np.sqrt(np.sum(np.abs(smaps) ** 2, axis=0)).astype(np.float32)
    return (smaps / (sos + np.finfo(np.float32).eps)[None]).astype(np.complex64)


def run_recon(smaps, y, idx, patch_sizes, strides, niters: int, sigma1=None, form: str = "tuned",
              index_base: int = 0, power_niter: int = 200, power_tol: float = 1e-6,
              restart_cutoff: float = 0.0, bsig: float = 1.0, return_components: bool = True,
              log_costs: bool = False):
    """Arguments are host numpy arrays or CUDA tensors in the layouts of
    :mod:`context`.  ``sigma1=None`` runs the power iteration (as
    σ1A_PRECOMPUTED = nothing, scripts/reconstruct.jl:152-158).

    Returns a dict with X (Ns,Nt,Nz,Ny,Nx), X_recon, restarts, lambdas,
    sigma1A and L, all on the host.  With ``log_costs`` it also returns
    dc_costs and reg_costs: the logger's (dc_cost, reg_cost) at X0 and after
    every iteration (scripts/reconstruct.jl:204-205, :227-230).
    """
    dev = torch.device("cuda")
    smaps_t = torch.as_tensor(smaps).to(dev, torch.complex64).contiguous()
    y_t = torch.as_tensor(y).to(dev, torch.complex64).contiguous()
    idx_t = torch.as_tensor(idx).to(dev, torch.int32).contiguous()
    Nc, Nz, Ny, Nx = smaps_t.shape
    Nt, _, K = y_t.shape
    with MSLRContext((Nx, Ny, Nz), Nc, Nt, K, patch_sizes, strides, form=form) as ctx:
        ctx.bind(smaps_t, y_t, idx_t, index_base=index_base)
        if sigma1 is None:
            sigma1, _ = ctx.power_iter(power_niter, power_tol)
        L = ctx.Ns * float(sigma1) ** 2
        X = ctx.init_x0()
        dcs, regs = [], []
        if log_costs:
            restarts, dcs, regs = ctx.pogm_run_costs(X, niters, L, restart_cutoff, bsig)
        else:
            restarts = ctx.pogm_run(X, niters, L, restart_cutoff, bsig)
        torch.cuda.synchronize()
        out = {
            "X_recon": X.sum(dim=0).cpu().numpy(),
            "restarts": restarts,
            "lambdas": list(ctx.lambdas),
            "sigma1A": float(sigma1),
            "L": L,
            "Nscales": ctx.Ns,
            "patch_sizes": ctx.patch_sizes,
            "strides": ctx.strides,
            "Niters": niters,
        }
        if log_costs:
            out["dc_costs"] = dcs
            out["reg_costs"] = regs
        if return_components:
            out["X"] = X.cpu().numpy()
    return out


def run_recon_kspace(ksp, smaps_raw, patch_sizes, strides, niters: int, sigma1=None, form: str = "tuned",
                     power_niter: int = 200, power_tol: float = 1e-6, restart_cutoff: float = 0.0,
                     bsig: float = 1.0, log_costs: bool = False):
    """run_recon from its raw inputs (scripts/reconstruct.jl:86-226): the
    zero-filled k-space ksp (Nt, Nc, Nz, Ny, Nx) and raw coil maps
    (Nc, Nz, Ny, Nx).  Maps normalisation, the 99th-percentile scaling, the
    sampling mask and its checks and the sample gathering run on the device
    (``MSLRContext.prepare``); then σ₁, X0 and POGM as :func:`run_recon`.
    Returns its dict plus ``scale_factor``, ``omega_counts`` (K) and the
    device-prepared ``smaps``, ``y`` and ``idx`` on the host; with
    ``log_costs`` also the logger's dc_costs and reg_costs as run_recon."""
    from .context import sampling
    dev = torch.device("cuda")
    ksp_t = torch.as_tensor(ksp).to(dev, torch.complex64).contiguous()
    sm_t = torch.as_tensor(smaps_raw).to(dev, torch.complex64).contiguous()
    Nt, Nc, Nz, Ny, Nx = ksp_t.shape
    K = sampling(ksp_t)
    with MSLRContext((Nx, Ny, Nz), Nc, Nt, K, patch_sizes, strides, form=form) as ctx:
        smaps, y, idx, scale = ctx.prepare(ksp_t, sm_t)
        if sigma1 is None:
            sigma1, _ = ctx.power_iter(power_niter, power_tol)
        L = ctx.Ns * float(sigma1) ** 2
        X = ctx.init_x0()
        costs = {}
        if log_costs:
            restarts, costs["dc_costs"], costs["reg_costs"] = ctx.pogm_run_costs(X, niters, L, restart_cutoff,
                                                                                 bsig)
        else:
            restarts = ctx.pogm_run(X, niters, L, restart_cutoff, bsig)
        torch.cuda.synchronize()
        return {
            **costs,
            "X_recon": X.sum(dim=0).cpu().numpy(),
            "X": X.cpu().numpy(),
            "restarts": restarts,
            "lambdas": list(ctx.lambdas),
            "sigma1A": float(sigma1),
            "L": L,
            "scale_factor": scale,
            "omega_counts": K,
            "smaps": smaps.cpu().numpy(),
            "y": y.cpu().numpy(),
            "idx": idx.cpu().numpy(),
            "Niters": niters,
        }


def run_recon_files(fn_ksp: str, fn_smaps: str, fn_recon_base: str, N, Nvc: int, Nt: int, PATCH_SIZES,
                    STRIDES, NITERS: int, sigma1A_precomputed=None, form: str = "tuned", nthreads: int = 0,
                    compress: bool = True):
    """run_recon(; fn_ksp, fn_smaps, fn_recon_base, N, Nvc, Nt, PATCH_SIZES,
    STRIDES, NITERS, σ1A_PRECOMPUTED, use_gpu=true) of scripts/reconstruct.jl:
    58-263, files included.

    Reads ``smaps`` with matread (:88) and ``ksp_epi_zf`` with h5read (:95),
    checks the k-space shape as the reference asserts (:97), runs the
    reconstruction on the device (:100-235, :func:`run_recon_kspace` with
    cost logging) and saves ``fn_recon_base * "_<Ns>scales.mat"`` with the
    reference's sixteen variables (:242-260) through matwrite.  Array dims
    follow the reference's Julia arrays (so X is MATLAB (Nx,Ny,Nz,Nt,Ns)).
    Returns the output path and the result dict (with ``seconds``: the wall
    time of reading, reconstructing and writing)."""
    import time
    from .matio import h5read, matread, matwrite
    t0 = time.perf_counter()
    Nx, Ny, Nz = (int(v) for v in N)
    smaps_raw = np.asarray(matread(fn_smaps, nthreads)["smaps"])
    ksp = h5read(fn_ksp, "ksp_epi_zf", nthreads)
    if ksp.shape != (Nt, Nvc, Nz, Ny, Nx):
        raise ValueError(f"Unexpected k-space shape: {tuple(reversed(ksp.shape))}")
    if smaps_raw.shape != (Nvc, Nz, Ny, Nx):
        raise ValueError(f"Unexpected coil-map shape: {tuple(reversed(smaps_raw.shape))}")
    t1 = time.perf_counter()
    out = run_recon_kspace(ksp.astype(np.complex64, copy=False), smaps_raw.astype(np.complex64, copy=False),
                           PATCH_SIZES, STRIDES, NITERS, sigma1=sigma1A_precomputed, form=form, log_costs=True)
    del ksp
    t2 = time.perf_counter()
    # Ω (Nx, Ny, Nz, Nt) from the per-frame sample indices, R from frame 1 (:108-109)
    omega = np.zeros((Nt, Nz * Ny * Nx), dtype=np.bool_)
    omega[np.arange(Nt)[:, None], out["idx"].astype(np.int64)] = True
    omega = omega.reshape(Nt, Nz, Ny, Nx)
    R = float(Nx * Ny * Nz) / float(omega[0].sum())
    Ns = len(PATCH_SIZES)
    fn_out = f"{fn_recon_base}_{Ns}scales.mat"
    matwrite(fn_out, {
        "X": out["X"],
        "X_recon": out["X_recon"],
        "omega": omega,
        "dc_costs": np.asarray(out["dc_costs"], dtype=np.float64),
        "reg_costs": np.asarray(out["reg_costs"], dtype=np.float64),
        "restarts": np.asarray(out["restarts"], dtype=np.bool_),
        "R": R,
        "sigma1A": float(out["sigma1A"]),
        "L": float(out["L"]),
        "Nscales": Ns,
        "patch_sizes": [np.asarray(p, dtype=np.int64) for p in PATCH_SIZES],
        "strides": [np.asarray(p, dtype=np.int64) for p in STRIDES],
        "lambdas": np.asarray(out["lambdas"], dtype=np.float64),
        "Niters": int(NITERS),
        "scale_factor": np.float32(out["scale_factor"]),
        "used_gpu": True,
    }, compress=compress, nthreads=nthreads)
    out["omega"] = omega
    out["R"] = R
    out["seconds"] = {"read": t1 - t0, "reconstruct": t2 - t1, "write": time.perf_counter() - t2}
    return fn_out, out
