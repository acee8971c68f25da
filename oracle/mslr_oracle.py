"""CPU oracle for the MSLR POGM hot path — TEST INFRASTRUCTURE ONLY.

This module restates, in numpy, the arithmetic of rextlfung/mslr-recon's
per-iteration path so that the CUDA library can be checked against it.  It is
imported only by ``tests/``, by ``__graft_entry__.smoke()`` and by the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``; the product path
(``mslr-recon_b200``) never imports it and fails loudly when its CUDA library
is missing.

Parity status: UNPINNED.  The reference is Julia (FFTW / LAPACK / CUDA.jl) and
ships no tests, golden vectors or fixtures; Julia is not installed here, so the
reference itself cannot be run to pin this restatement.  The restatement is
instead checked against known-answer properties of the mathematics (unitary
SENSE adjointness, SVST of matrices with known SVD, patch extract/recombine
identities, Ong–Lustig λ values) in ``tests/test_oracle.py``.

Memory layouts follow the reference's column-major Julia arrays exactly, read
as C-order numpy arrays with the axes reversed:

=====================  ==========================  ==========================
quantity               Julia (column-major)        numpy here (C-order)
=====================  ==========================  ==========================
image time series      (Nx, Ny, Nz, Nt)            (Nt, Nz, Ny, Nx)
multi-scale X          (Nx, Ny, Nz, Nt, Ns)        (Ns, Nt, Nz, Ny, Nx)
coil maps              (Nx, Ny, Nz, Nc)            (Nc, Nz, Ny, Nx)
sampled k-space y      (K, Nc, Nt)                 (Nt, Nc, K)
patch stack P          (p, Nt, Np)                 (Np, Nt, p)
=====================  ==========================  ==========================

Linear k-space indices are the reference's ``findall(vec(samp))`` minus one:
ascending 0-based column-major indices ``x + Nx*(y + Ny*z)``, i.e. flat
indices into a C-order ``(Nz, Ny, Nx)`` array.

Every function cites the reference file:line it restates.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass
from typing import Callable, List, Sequence

import numpy as np
import scipy.fft as sfft
import scipy.linalg as sla

SPATIAL_AXES = (-3, -2, -1)


# ---------------------------------------------------------------------------
# Patch geometry — src/recon.jl:53-78 (img2patches), :96-126 (patches2img)
# ---------------------------------------------------------------------------
def cld(a: int, b: int) -> int:
    """Julia ``cld`` (ceiling division) for integers."""
    return -((-a) // b)


@dataclass(frozen=True)
class PatchGeometry:
    """Clamped-stride patch grid of one scale (src/recon.jl:57-75).

    ``ps`` / ``ss`` / ``N`` are (x, y, z) triples.  ``starts[d]`` holds the
    0-based start of every patch along dimension d; patch ``ip`` (0-based)
    enumerates ix fastest, then iy, then iz (src/recon.jl:69).
    """

    N: tuple
    ps: tuple
    ss: tuple
    nsteps: tuple
    starts: tuple

    @property
    def Np(self) -> int:
        return (self.nsteps[0] + 1) * (self.nsteps[1] + 1) * (self.nsteps[2] + 1)

    @property
    def p(self) -> int:
        return self.ps[0] * self.ps[1] * self.ps[2]

    def patch_start(self, ip: int) -> tuple:
        nx, ny = self.nsteps[0] + 1, self.nsteps[1] + 1
        ix = ip % nx
        iy = (ip // nx) % ny
        iz = ip // (nx * ny)
        return (self.starts[0][ix], self.starts[1][iy], self.starts[2][iz])


def patch_geometry(N: Sequence[int], patch_size: Sequence[int], stride_size: Sequence[int]) -> PatchGeometry:
    """src/recon.jl:54-72: ``ps = min(ps, N)``, ``nsteps = cld(N-ps, ss)``,
    ``start(i) = min(i*ss + 1, N - ps + 1)`` (1-based; returned 0-based)."""
    N = tuple(int(v) for v in N)
    ps = tuple(min(int(p), n) for p, n in zip(patch_size, N))
    ss = tuple(int(s) for s in stride_size)
    if any(s <= 0 for s in ss):
        raise ValueError("strides must be positive")
    nsteps = tuple(cld(n - p, s) for n, p, s in zip(N, ps, ss))
    starts = tuple(
        tuple(min(i * s, n - p) for i in range(ns + 1))
        for n, p, s, ns in zip(N, ps, ss, nsteps)
    )
    return PatchGeometry(N=N, ps=ps, ss=ss, nsteps=nsteps, starts=starts)


def img2patches(img: np.ndarray, patch_size, stride_size) -> np.ndarray:
    """src/recon.jl:53-78.  ``img`` (Nt, Nz, Ny, Nx) -> P (Np, Nt, p)."""
    Nt, Nz, Ny, Nx = img.shape
    g = patch_geometry((Nx, Ny, Nz), patch_size, stride_size)
    psx, psy, psz = g.ps
    P = np.zeros((g.Np, Nt, g.p), dtype=img.dtype)
    for ip in range(g.Np):
        sx, sy, sz = g.patch_start(ip)
        blk = img[:, sz:sz + psz, sy:sy + psy, sx:sx + psx]
        P[ip] = blk.reshape(Nt, g.p)
    return P


def patches2img(P: np.ndarray, patch_size, stride_size, og_size) -> np.ndarray:
    """src/recon.jl:96-126: sum patches in ascending ip, Float32 coverage
    count, ``max(count, 1)``, divide."""
    Np, Nt, p = P.shape
    g = patch_geometry(og_size, patch_size, stride_size)
    Nx, Ny, Nz = g.N
    psx, psy, psz = g.ps
    img = np.zeros((Nt, Nz, Ny, Nx), dtype=P.dtype)
    count = np.zeros((Nz, Ny, Nx), dtype=np.float32)
    for ip in range(Np):
        sx, sy, sz = g.patch_start(ip)
        img[:, sz:sz + psz, sy:sy + psy, sx:sx + psx] += P[ip].reshape(Nt, psz, psy, psx)
        count[sz:sz + psz, sy:sy + psy, sx:sx + psx] += np.float32(1)
    count = np.maximum(count, np.float32(1))
    # Julia's ComplexF32 ./ Float32 divides the real and imaginary parts
    # separately (not a complex division)
    c = count[None].astype(img.real.dtype)
    img.real /= c
    img.imag /= c
    return img


def coverage_count(N, patch_size, stride_size) -> np.ndarray:
    """Float32 coverage counts before the ``max(.,1)`` clamp
    (src/recon.jl:113-121)."""
    g = patch_geometry(N, patch_size, stride_size)
    Nx, Ny, Nz = g.N
    psx, psy, psz = g.ps
    count = np.zeros((Nz, Ny, Nx), dtype=np.float32)
    for ip in range(g.Np):
        sx, sy, sz = g.patch_start(ip)
        count[sz:sz + psz, sy:sy + psy, sx:sx + psx] += np.float32(1)
    return count


# ---------------------------------------------------------------------------
# SVST — src/recon.jl:183-211, loops :217-269
# ---------------------------------------------------------------------------
def _svd(X: np.ndarray):
    """gesdd with a gesvd fallback, as src/recon.jl:189-193.  numpy's thin SVD
    is LAPACK gesdd and runs without the interpreter lock, so patches in a
    thread pool run concurrently; scipy's gesvd is the fallback."""
    try:
        return np.linalg.svd(X, full_matrices=False)
    except (np.linalg.LinAlgError, ValueError):
        return sla.svd(X, full_matrices=False, lapack_driver="gesvd", check_finite=False)


def svst(X: np.ndarray, beta: float) -> np.ndarray:
    """src/recon.jl:183-205: zero-norm skip, thin SVD, ``max(S - β, 0)``,
    rebuild from the kept (s > 0) columns (CPU variant)."""
    if np.linalg.norm(X) == 0:
        return np.zeros_like(X)
    U, S, Vt = _svd(X)
    s = np.maximum(S - S.dtype.type(beta), 0)
    keep = s > 0
    if not keep.any():
        return np.zeros_like(X)
    return (U[:, keep] * s[keep]) @ Vt[keep, :]


def patch_svst(img: np.ndarray, beta, patch_size, stride_size) -> np.ndarray:
    """src/recon.jl:251-256 (global β) and :263-268 (per-patch λs).

    ``img`` (Nt, Nz, Ny, Nx).  Each patch matrix is (p × Nt) in the
    reference; here P[ip] is its transpose (Nt × p), and SVST commutes with
    transposition, so ``svst(P[ip].T).T`` is applied.
    """
    Nt, Nz, Ny, Nx = img.shape
    P = img2patches(img, patch_size, stride_size)
    Np = P.shape[0]
    betas = np.broadcast_to(np.asarray(beta, dtype=np.float64), (Np,))
    for ip in range(Np):
        P[ip] = svst(P[ip].T.copy(), float(betas[ip])).T
    return patches2img(P, patch_size, stride_size, (Nx, Ny, Nz))


def patch_nucnorm(P: np.ndarray) -> float:
    """src/recon.jl:138-146: Σ over patches of Σ svdvals (Float64 sum)."""
    total = 0.0
    for ip in range(P.shape[0]):
        total += float(np.sum(sla.svdvals(P[ip], check_finite=False), dtype=np.float64))
    return total


def patch_nucnorm_weighted(P: np.ndarray, lams) -> float:
    """src/recon.jl:154-166: Σ over patches of λ_p · Σ svdvals (0 for a zero
    patch), divided by the number of patches."""
    total = 0.0
    for ip in range(P.shape[0]):
        s = np.linalg.svd(P[ip], compute_uv=False)
        total += float(lams[ip]) * float(np.sum(s, dtype=np.float64)) if s[0] > 0 else 0.0
    return total / P.shape[0]


# ---------------------------------------------------------------------------
# SENSE operator — src/sense_gpu.jl:51-101 (convention of MIRT.Asense with
# fft_forward=true, unitary=true).  The adjoint is the exact adjoint of the
# forward (scale·bfft), i.e. MIRT's unitary pair.
# ---------------------------------------------------------------------------
def _fftc(x, workers):
    return sfft.fftshift(sfft.fftn(sfft.ifftshift(x, axes=SPATIAL_AXES), axes=SPATIAL_AXES,
                                    workers=workers), axes=SPATIAL_AXES)


def _bfftc(k, workers):
    """Exact adjoint of :func:`_fftc`: fftshift(bfft(ifftshift(k))).  The
    reference writes ifftshift(ifft(fftshift(.))) (src/sense_gpu.jl:93), which
    is the same map for the even sizes it is used with."""
    n = int(np.prod(k.shape[-3:]))
    # unnormalised inverse: ifft * n
    return sfft.fftshift(sfft.ifftn(sfft.ifftshift(k, axes=SPATIAL_AXES), axes=SPATIAL_AXES,
                                    workers=workers), axes=SPATIAL_AXES) * n


def sense_forward_frame(x: np.ndarray, smaps: np.ndarray, idx: np.ndarray, workers: int = -1) -> np.ndarray:
    """src/sense_gpu.jl:71-81: ``scale·fftshift(fft(ifftshift(S.*x)))[idx, :]``.

    x (Nz, Ny, Nx); smaps (Nc, Nz, Ny, Nx); idx 0-based ascending (K,).
    Returns (Nc, K)."""
    Nc = smaps.shape[0]
    n = x.size
    scale = 1.0 / math.sqrt(n)
    kc = _fftc(smaps * x[None], workers) * scale
    return kc.reshape(Nc, -1)[:, idx]


def sense_adjoint_frame(y: np.ndarray, smaps: np.ndarray, idx: np.ndarray, workers: int = -1) -> np.ndarray:
    """Exact adjoint of :func:`sense_forward_frame` (src/sense_gpu.jl:84-101
    with the unitary ``scale·bfft`` inverse).  y (Nc, K) -> (Nz, Ny, Nx)."""
    Nc, Nz, Ny, Nx = smaps.shape
    n = Nx * Ny * Nz
    scale = 1.0 / math.sqrt(n)
    full = np.zeros((Nc, n), dtype=np.result_type(y.dtype, smaps.dtype))
    full[:, idx] = y
    xc = _bfftc(full.reshape(Nc, Nz, Ny, Nx), workers) * scale
    return np.sum(np.conj(smaps) * xc, axis=0)


def sense_forward(x: np.ndarray, smaps: np.ndarray, idx: np.ndarray, workers: int = -1) -> np.ndarray:
    """Block-diagonal over frames (scripts/reconstruct.jl:142-147).
    x (Nt, Nz, Ny, Nx); idx (Nt, K) -> y (Nt, Nc, K)."""
    return np.stack([sense_forward_frame(x[t], smaps, idx[t], workers) for t in range(x.shape[0])])


def sense_adjoint(y: np.ndarray, smaps: np.ndarray, idx: np.ndarray, workers: int = -1) -> np.ndarray:
    return np.stack([sense_adjoint_frame(y[t], smaps, idx[t], workers) for t in range(y.shape[0])])


def normal_op(x: np.ndarray, smaps: np.ndarray, idx: np.ndarray, workers: int = -1) -> np.ndarray:
    """A'A x per frame (no data term)."""
    return sense_adjoint(sense_forward(x, smaps, idx, workers), smaps, idx, workers)


# ---------------------------------------------------------------------------
# POGM — src/mirt_mod.jl:26-29 (_gr_restart), :74-188 (pogm_mod)
# ---------------------------------------------------------------------------
def _gr_restart(Fgrad, ynew_yold, restart_cutoff) -> bool:
    """src/mirt_mod.jl:26-29: ``sum(Float64, real(-Fgrad .* ynew_yold)) <=
    cutoff * norm(Fgrad) * norm(ynew_yold)`` — an unconjugated product."""
    lhs = float(np.sum(np.real(-Fgrad * ynew_yold), dtype=np.float64))
    rhs = restart_cutoff * float(np.linalg.norm(Fgrad)) * float(np.linalg.norm(ynew_yold))
    return lhs <= rhs


def pogm_mod(x0, Fcost: Callable, f_grad: Callable, f_L: float, *, f_mu: float = 0.0,
             mom: str = "pogm", restart: str = "gr", restart_cutoff: float = 0.0,
             bsig: float = 1.0, niter: int = 10,
             g_prox: Callable = lambda z, c: z,
             fun: Callable = lambda it, xk, yk, r: None,
             iter_callback: Callable | None = None):
    """Line-by-line restatement of src/mirt_mod.jl:74-188.

    Object identity is preserved on purpose: when ``g_prox`` mutates and
    returns its argument (as the reference's g_prox does,
    scripts/reconstruct.jl:196-202), ``xnew is znew`` and the
    ``β·α/ζold·(xold − zold)`` term vanishes exactly as in the reference.
    ``iter_callback(iter, xnew, is_restart)`` is an oracle-only hook used by the
    per-iteration parity tests.
    """
    if mom not in ("pgm", "fpgm", "pogm"):
        raise ValueError(f"mom={mom}")
    if restart not in ("none", "gr", "fr"):
        raise ValueError(f"restart={restart}")
    if f_L < 0 or f_mu < 0 or bsig < 0 or not abs(restart_cutoff) < 1:
        raise ValueError("bad pogm_mod argument")
    L = f_L
    mu = f_mu
    q = mu / L
    told = 1.0
    sig = 1.0
    zetaold = 1.0
    xold = x0
    yold = x0
    uold = x0
    zold = x0
    Fcostold = Fcost(x0)
    Fgradold = np.zeros(np.shape(x0))
    out = [None] * (niter + 1)
    out[0] = fun(0, x0, x0, False)
    xnew = ynew = None
    for it in range(1, niter + 1):
        alpha = 2 / (L + mu) if (mom == "pgm" and mu != 0) else 1 / L
        fgrad = f_grad(xold)
        is_restart = False
        if mom in ("pgm", "fpgm"):
            ynew = g_prox(xold - alpha * fgrad, alpha)
            Fgrad = -(1 / alpha) * (ynew - xold)
            Fcostnew = Fcost(ynew)
            if restart != "none":
                if (restart == "fr" and Fcostnew > Fcostold) or \
                   (restart == "gr" and _gr_restart(Fgrad, ynew - yold, restart_cutoff)):
                    told = 1.0
                    is_restart = True
                Fcostold = Fcostnew
        else:
            unew = xold - alpha * fgrad
        if mom == "fpgm" and mu != 0:
            beta = (1 - math.sqrt(q)) / (1 + math.sqrt(q))
        elif mom == "pogm" and mu != 0:
            beta = (2 + q - math.sqrt(q ** 2 + 8 * q)) ** 2 / 4 / (1 - q)
        elif mom != "pgm":
            if mom == "pogm" and it == niter:
                tnew = 0.5 * (1 + math.sqrt(1 + 8 * told ** 2))
            else:
                tnew = 0.5 * (1 + math.sqrt(1 + 4 * told ** 2))
            beta = (told - 1) / tnew
        if mom == "pgm":
            xnew = ynew
        elif mom == "fpgm":
            xnew = ynew + beta * (ynew - yold)
        else:
            gamma = (2 + q - math.sqrt(q ** 2 + 8 * q)) / 2 if mu != 0 else sig * told / tnew
            znew = unew + beta * (unew - uold) + gamma * (unew - xold) \
                - beta * alpha / zetaold * (xold - zold)
            zetanew = alpha * (1 + beta + gamma)
            xnew = g_prox(znew, zetanew)
            Fgrad = fgrad - (1 / zetanew) * (xnew - znew)
            ynew = xold - alpha * Fgrad
            Fcostnew = Fcost(xnew)
            if restart != "none":
                if (restart == "fr" and Fcostnew > Fcostold) or \
                   (restart == "gr" and _gr_restart(Fgrad, ynew - yold, restart_cutoff)):
                    tnew = 1.0
                    sig = 1.0
                    is_restart = True
                elif float(np.sum(np.real(Fgrad * Fgradold), dtype=np.float64)) < 0:
                    sig = bsig * sig
                Fcostold = Fcostnew
                Fgradold = Fgrad
            uold = unew
            zold = znew
            zetaold = zetanew
        out[it] = fun(it, xnew, ynew, is_restart)
        if iter_callback is not None:
            iter_callback(it, xnew, is_restart)
        xold = xnew
        yold = ynew
        if mom != "pgm" and mu == 0:
            told = tnew
    return (xnew if mom == "pogm" else ynew), out


# ---------------------------------------------------------------------------
# Power iteration — src/mirt_mod.jl:215-238
# ---------------------------------------------------------------------------
def poweriter_mod(Aop: Callable, Aadj: Callable, x0: np.ndarray, niter: int = 200,
                  tol: float = 1e-6):
    """src/mirt_mod.jl:215-238 with ``x0 = ones``.  Returns (x, σ1)."""
    x = x0.copy()
    ratio_old = math.inf
    for _ in range(niter):
        Ax = Aop(x)
        ratio = float(np.linalg.norm(Ax)) / float(np.linalg.norm(x))
        if abs(ratio - ratio_old) / ratio < tol:
            break
        ratio_old = ratio
        x = Aadj(Ax)
        x = x / np.linalg.norm(x)
    return x, float(np.linalg.norm(Aop(x))) / float(np.linalg.norm(x))


# ---------------------------------------------------------------------------
# λ_k and L — scripts/reconstruct.jl:159, :163-169
# ---------------------------------------------------------------------------
def ong_lustig_lambdas(N, Nt, patch_sizes) -> List[float]:
    """scripts/reconstruct.jl:163-169 (uses the *unclamped* patch sizes)."""
    nvox = int(np.prod(N))
    out = []
    for ps in patch_sizes:
        p = int(np.prod(ps))
        out.append(math.sqrt(p) + math.sqrt(Nt) + math.sqrt(math.log(nvox * Nt / max(p, Nt))))
    return out


# ---------------------------------------------------------------------------
# run_recon's closures — scripts/reconstruct.jl:174-214, pogm call :220-226
# ---------------------------------------------------------------------------
@dataclass
class ReconProblem:
    smaps: np.ndarray          # (Nc, Nz, Ny, Nx), SOS-normalised
    idx: np.ndarray            # (Nt, K) 0-based
    y: np.ndarray              # (Nt, Nc, K)
    patch_sizes: list
    strides: list
    sigma1: float = 1.0
    workers: int = -1

    @property
    def N(self):
        Nc, Nz, Ny, Nx = self.smaps.shape
        return (Nx, Ny, Nz)

    @property
    def Nt(self):
        return self.y.shape[0]

    @property
    def Ns(self):
        return len(self.patch_sizes)

    def lambdas(self):
        return ong_lustig_lambdas(self.N, self.Nt, self.patch_sizes)

    def lipschitz(self):
        return self.Ns * self.sigma1 ** 2


def run_recon_arrays(prob: ReconProblem, niters: int, dtype=np.complex128, log_costs: bool = False,
                     iter_callback=None, restart_cutoff: float = 0.0, bsig: float = 1.0,
                     mom: str = "pogm", restart: str = "gr", f_mu: float = 0.0):
    """The hot loop of scripts/reconstruct.jl:174-226 on in-memory arrays.

    ``dtype=np.complex128`` is the FP64 oracle; ``np.complex64`` mimics the
    reference CPU precision.  Returns (X, restarts, dc_costs, reg_costs);
    the cost lists are empty unless ``log_costs``.  ``mom``, ``restart`` and
    ``f_mu`` are pogm_mod's options (run_recon passes :pogm, :gr, 0); Fcost
    is run_recon's comp_cost = dc_cost + reg_cost, evaluated by pogm_mod
    only where a restart rule reads it (restart = "fr").
    """
    Nx, Ny, Nz = prob.N
    Nt, Ns = prob.Nt, prob.Ns
    smaps = prob.smaps.astype(dtype)
    y = prob.y.astype(dtype)
    idx = prob.idx
    lam = prob.lambdas()
    L = prob.lipschitz()
    w = prob.workers

    def image_sum(X):
        return X.sum(axis=0)

    def dc_cost(X):
        r = sense_forward(image_sum(X), smaps, idx, w) - y
        return 0.5 * float(np.linalg.norm(r)) ** 2

    def dc_cost_grad(X):
        g = sense_adjoint(sense_forward(image_sum(X), smaps, idx, w) - y, smaps, idx, w)
        return np.broadcast_to(g[None], (Ns,) + g.shape).astype(dtype, copy=True)

    def reg_cost(X):
        return sum(lam[k] * patch_nucnorm(img2patches(X[k], prob.patch_sizes[k], prob.strides[k]))
                   for k in range(Ns))

    def g_prox(X, c):
        for k in range(Ns):
            X[k] = patch_svst(X[k], c * lam[k], prob.patch_sizes[k], prob.strides[k])
        return X

    restarts = []
    dcs, regs = [], []

    def logger(it, xk, yk, is_restart):
        restarts.append(bool(is_restart))
        if log_costs:
            dcs.append(dc_cost(xk))
            regs.append(reg_cost(xk))
        return None

    X0 = np.zeros((Ns, Nt, Nz, Ny, Nx), dtype=dtype)
    X0[0] = sense_adjoint(y, smaps, idx, w)
    fcost = (lambda X: dc_cost(X) + reg_cost(X)) if restart == "fr" else (lambda X: 0.0)
    Xf, _ = pogm_mod(X0, fcost, dc_cost_grad, L, mom=mom, restart=restart, f_mu=f_mu, niter=niters,
                     g_prox=g_prox, fun=logger, iter_callback=iter_callback,
                     restart_cutoff=restart_cutoff, bsig=bsig)
    return Xf, restarts, dcs, regs


# ---------------------------------------------------------------------------
# Full-size runs (the benchmark's 90×90×60 workloads).  The same arithmetic as
# run_recon_arrays — per-frame SENSE of src/sense_gpu.jl:71-101, per-patch
# gesdd SVST of src/recon.jl:183-211 with the ascending-ip recombine of
# :96-126, and pogm_mod's aliased recurrence (src/mirt_mod.jl:144-176 with
# run_recon's in-place g_prox, scripts/reconstruct.jl:196-202) — organised
# for host memory and cores: frames, patches and update chunks are spread
# over a thread pool (as the reference's @threads over patches), patches are
# extracted and recombined one at a time instead of as a whole patch stack,
# and the recurrence is written out with the aliasing resolved (xold is
# zold, so the β·α/ζold·(xold − zold) term is zero, Fgrad = fgrad and
# ynew = unew) and evaluated in place.  tests/test_oracle.py pins it to
# run_recon_arrays.
# ---------------------------------------------------------------------------
def _pool_map(pool, fn, items, window: int = 256):
    """Ordered map over ``items`` with at most ``window`` tasks in flight."""
    items = list(items)
    for i0 in range(0, len(items), window):
        yield from pool.map(fn, items[i0:i0 + window])


class _ShiftedSense:
    """sense_forward_frame / sense_adjoint_frame with the centring shifts
    moved onto the coil maps and the sample indices.  For even image sizes
    fftshift and ifftshift are the same permutation p of the grid, an
    involution, so fftshift(fft(ifftshift(S·x)))[idx] = fft(pS · px)[p(idx)]
    and Σ_c conj(S_c)·fftshift(Y_c) = fftshift(Σ_c conj(pS_c)·Y_c): the same
    products and sums on permuted arrays (equal to the plain functions up to
    the FFT library's FP64 rounding, which depends on memory layout), with
    the shifted maps made once instead of every frame's coil images shifted
    twice.  Odd sizes use the plain functions."""

    def __init__(self, smaps: np.ndarray):
        self.smaps = smaps
        Nc, Nz, Ny, Nx = smaps.shape
        self.even = Nz % 2 == 0 and Ny % 2 == 0 and Nx % 2 == 0
        self.n = Nx * Ny * Nz
        self.scale = 1.0 / math.sqrt(self.n)
        if self.even:
            self.ps = sfft.ifftshift(smaps, axes=SPATIAL_AXES)
            self.pc = np.conj(self.ps)
            self.perm = sfft.ifftshift(np.arange(self.n).reshape(Nz, Ny, Nx)).reshape(-1)

    def forward(self, x: np.ndarray, idx: np.ndarray) -> np.ndarray:
        if not self.even:
            return sense_forward_frame(x, self.smaps, idx, 1)
        Nc = self.ps.shape[0]
        k = sfft.fftn(self.ps * sfft.ifftshift(x)[None], axes=SPATIAL_AXES, workers=1, overwrite_x=True)
        return k.reshape(Nc, -1)[:, self.perm[idx]] * self.scale

    def adjoint(self, y: np.ndarray, idx: np.ndarray) -> np.ndarray:
        if not self.even:
            return sense_adjoint_frame(y, self.smaps, idx, 1)
        Nc, Nz, Ny, Nx = self.ps.shape
        full = np.zeros((Nc, self.n), dtype=np.result_type(y.dtype, self.ps.dtype))
        full[:, self.perm[idx]] = y
        xc = sfft.ifftn(full.reshape(Nc, Nz, Ny, Nx), axes=SPATIAL_AXES, workers=1, overwrite_x=True)
        xc *= self.n
        xc *= self.scale
        return sfft.fftshift(np.sum(self.pc * xc, axis=0))


def dc_grad_frames(X: np.ndarray, smaps: np.ndarray, y: np.ndarray, idx: np.ndarray, pool,
                   out: np.ndarray | None = None, sense: _ShiftedSense | None = None) -> np.ndarray:
    """dc_cost_grad before the repeat (scripts/reconstruct.jl:180-183),
    g[t] = A_t'(A_t Σ_k X[k, t] − y[t]), frames in parallel."""
    Ns, Nt = X.shape[:2]
    g = np.empty(X.shape[1:], dtype=X.dtype) if out is None else out
    sense = sense or _ShiftedSense(smaps)

    def frame(t):
        xs = X[0, t].copy()
        for k in range(1, Ns):
            xs += X[k, t]
        r = sense.forward(xs, idx[t]) - y[t]
        g[t] = sense.adjoint(r, idx[t])
        return t

    for _ in _pool_map(pool, frame, range(Nt)):
        pass
    return g


def adjoint_frames(y: np.ndarray, smaps: np.ndarray, idx: np.ndarray, pool,
                   sense: _ShiftedSense | None = None) -> np.ndarray:
    """A'y frame by frame in parallel (X0 of scripts/reconstruct.jl:209-214)."""
    Nt = y.shape[0]
    Nc, Nz, Ny, Nx = smaps.shape
    out = np.empty((Nt, Nz, Ny, Nx), dtype=np.result_type(y.dtype, smaps.dtype))
    sense = sense or _ShiftedSense(smaps)

    def frame(t):
        out[t] = sense.adjoint(y[t], idx[t])
        return t

    for _ in _pool_map(pool, frame, range(Nt)):
        pass
    return out


def patch_svst_inplace(img: np.ndarray, beta: float, patch_size, stride_size, pool,
                       blas_threads: int = 1) -> np.ndarray:
    """patch_svst (src/recon.jl:251-256) into ``img`` itself, one patch at a
    time: SVST of every patch of the input, sums in ascending ip, FP32
    coverage count clamped to 1, component-wise division.  A single-patch
    scale runs its one SVD with ``blas_threads`` BLAS threads."""
    Nt, Nz, Ny, Nx = img.shape
    g = patch_geometry((Nx, Ny, Nz), patch_size, stride_size)
    psx, psy, psz = g.ps

    def block(ip):
        sx, sy, sz = g.patch_start(ip)
        return (slice(None), slice(sz, sz + psz), slice(sy, sy + psy), slice(sx, sx + psx))

    def one(ip):
        P = img[block(ip)].reshape(Nt, g.p)
        return svst(P.T.copy(), beta).T.reshape(Nt, psz, psy, psx)

    out = np.zeros_like(img)
    if g.Np == 1:
        from threadpoolctl import threadpool_limits
        with threadpool_limits(blas_threads, "blas"):
            res = one(0)
        out[block(0)] += res
        del res
    else:
        for ip, res in zip(range(g.Np), _pool_map(pool, one, range(g.Np))):
            out[block(ip)] += res
    cnt = coverage_count((Nx, Ny, Nz), patch_size, stride_size)
    c = np.maximum(cnt, np.float32(1)).astype(img.real.dtype)
    out.real /= c[None]
    out.imag /= c[None]
    img[...] = out
    return img


def run_recon_large(prob: ReconProblem, niters: int, iter_callback=None, threads: int | None = None,
                    restart_cutoff: float = 0.0, bsig: float = 1.0, chunk: int = 1 << 20,
                    log: Callable | None = None):
    """run_recon_arrays in FP64 for full-size problems.  Returns (X, restarts);
    ``iter_callback(it, X, is_restart)`` sees X after every iteration (X is
    overwritten by the next one); ``log(phase, seconds)`` receives the time of
    every phase."""
    import time
    from concurrent.futures import ThreadPoolExecutor
    threads = threads or os.cpu_count() or 1
    clock = [time.perf_counter()]

    def lap(phase):
        if log is not None:
            t = time.perf_counter()
            log(phase, t - clock[0])
            clock[0] = t

    Nx, Ny, Nz = prob.N
    Nt, Ns = prob.Nt, prob.Ns
    dtype = np.complex128
    smaps = prob.smaps.astype(dtype)
    y = prob.y.astype(dtype)
    idx = prob.idx
    lam = prob.lambdas()
    L = prob.lipschitz()
    restarts = [False]
    sense = _ShiftedSense(smaps)
    with ThreadPoolExecutor(threads) as pool:
        x = np.zeros((Ns, Nt, Nz, Ny, Nx), dtype=dtype)
        x[0] = adjoint_frames(y, smaps, idx, pool, sense)
        lap("x0")
        uold = x.copy()                          # u_0 = y_0 = x_0
        g = np.empty((Nt, Nz, Ny, Nx), dtype=dtype)
        gold = np.zeros_like(g) if bsig != 1.0 else None
        u = np.empty_like(x)
        told, sig = 1.0, 1.0
        E = g.size
        xf, uf, of, gf = x.reshape(Ns, E), u.reshape(Ns, E), uold.reshape(Ns, E), g.reshape(E)
        for it in range(1, niters + 1):
            alpha = 1.0 / L
            dc_grad_frames(x, smaps, y, idx, pool, out=g, sense=sense)
            lap("dc_grad")
            tnew = 0.5 * (1 + math.sqrt(1 + (8 if it == niters else 4) * told ** 2))
            beta = (told - 1) / tnew
            gamma = sig * told / tnew

            # u = x − α g;  restart sums over u − uold;  z = u + β(u − uold) + γ(u − x) into x;
            # chunks in parallel, their partial sums added in chunk order
            def update(e0, xf=xf, uf=uf, of=of):
                sl = slice(e0, min(E, e0 + chunk))
                gs = gf[sl]
                part = [0.0, 0.0, float(np.vdot(gs, gs).real), 0.0]
                if gold is not None:
                    part[3] = float(np.sum(np.real(gs * gold.reshape(E)[sl]), dtype=np.float64))
                for k in range(Ns):
                    uk = xf[k, sl] - alpha * gs
                    du = uk - of[k, sl]
                    part[0] += float(np.sum(np.real(-gs * du), dtype=np.float64))
                    part[1] += float(np.vdot(du, du).real)
                    xf[k, sl] = uk + beta * du + gamma * (uk - xf[k, sl])
                    uf[k, sl] = uk
                return part

            dot, n_du, n_g, gg = 0.0, 0.0, 0.0, 0.0
            for p0, p1, p2, p3 in _pool_map(pool, update, range(0, E, chunk)):
                dot, n_du, n_g, gg = dot + p0, n_du + p1, n_g + p2, gg + p3
            lap("update")
            zeta = alpha * (1 + beta + gamma)
            for k in range(Ns):
                patch_svst_inplace(x[k], zeta * lam[k], prob.patch_sizes[k], prob.strides[k], pool,
                                   blas_threads=threads)
                lap(f"svst_{k}")
            # _gr_restart with Fgrad = the Ns-fold repeat of g, ynew − yold = u − uold
            rhs = restart_cutoff * math.sqrt(Ns * n_g) * math.sqrt(n_du)
            is_restart = dot <= rhs
            if is_restart:
                tnew, sig = 1.0, 1.0
            elif gold is not None and Ns * gg < 0:
                sig = bsig * sig
            if gold is not None:
                gold[...] = g
            restarts.append(bool(is_restart))
            u, uold = uold, u
            uf, of = of, uf
            told = tnew
            if iter_callback is not None:
                iter_callback(it, x, is_restart)
    return x, restarts


def rel_err_chunked(a: np.ndarray, b: np.ndarray, chunk: int = 1 << 22) -> float:
    """:func:`rel_err` of two large arrays without full-size FP64 copies."""
    af, bf = a.reshape(-1), b.reshape(-1)
    num = den = 0.0
    for e0 in range(0, af.size, chunk):
        d = af[e0:e0 + chunk].astype(np.complex128) - bf[e0:e0 + chunk]
        bb = bf[e0:e0 + chunk].astype(np.complex128)
        num += float(np.vdot(d, d).real)
        den += float(np.vdot(bb, bb).real)
    return math.sqrt(num) / (math.sqrt(den) if den > 0 else 1.0)


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """Relative Frobenius error ‖a − b‖ / ‖b‖ (FP64 accumulation)."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)


# ---------------------------------------------------------------------------
# Differentiation of the unrolled POGM with respect to log λ_k.
#
# The reference does not differentiate run_recon; this section restates the
# forward it does run (pogm_mod with mom=:pogm, restart=:gr and run_recon's
# aliasing g_prox, src/mirt_mod.jl:74-188, scripts/reconstruct.jl:196-202) as
# the explicit recurrence that aliasing reduces it to
#     u_i = x_{i-1} − α ∇f(x_{i-1})
#     z_i = (1 + β_i + γ_i) u_i − β_i u_{i-1} − γ_i x_{i-1},   u_0 = x_0
#     x_i = prox_{ζ_i}(z_i)       (per scale: patch SVST, threshold ζ_i λ_k)
# with the restart decisions and momentum scalars of the run held fixed
# (they are piecewise constant in λ), and differentiates
#     loss = ½ ‖Σ_k X_k − X_true‖²
# by reverse accumulation.  The patch-SVST backward uses the Gram form of
# SVST: for a patch matrix A (p × q, p ≥ q; otherwise applied to Aᴴ),
#     Y = A W,  W = f(G) = V f(Λ) Vᴴ,  G = Aᴴ A,  f(λ) = max(1 − β/√λ, 0),
#     Ā = Ȳ W + A K,   K = V (F ⊙ Vᴴ (W̄ + W̄ᴴ) V) Vᴴ,   W̄ = Aᴴ Ȳ,
#     ∂loss/∂β = Σ_i ∂f/∂β(λ_i) Re (Vᴴ W̄ V)_ii,
# F the divided differences of f (Daleckii–Krein).
# ---------------------------------------------------------------------------
def svst_divided_differences(lam: np.ndarray, beta: float):
    """(f(λ), ∂f/∂β(λ), F) for f(λ) = max(1 − β/√λ, 0) at the eigenvalues
    ``lam`` of a patch Gram matrix; F_ij = (f_i − f_j)/(λ_i − λ_j), f'(λ_i) on
    the diagonal, written without cancellation."""
    s = np.sqrt(np.maximum(lam, 0.0))
    above = s > beta
    f = np.where(above, 1.0 - beta / np.where(above, s, 1.0), 0.0)
    fb = np.where(above, -1.0 / np.where(above, s, 1.0), 0.0)
    si, sj = s[:, None], s[None, :]
    ai, aj = above[:, None], above[None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        both = beta / (si * sj * (si + sj))
        i_only = (si - beta) / (si * (si - sj) * (si + sj))
        j_only = (sj - beta) / (sj * (sj - si) * (si + sj))
    F = np.where(ai & aj, both, np.where(ai & ~aj, i_only, np.where(~ai & aj, j_only, 0.0)))
    return f, fb, F


def svst_vjp(A: np.ndarray, beta: float, Ybar: np.ndarray):
    """Cotangent of A and of β for Y = SVST(A, β) (src/recon.jl:183-211),
    given the cotangent Ybar of Y (real inner product Re tr(Xᴴ Y))."""
    if A.shape[0] < A.shape[1]:
        Abar, bb = svst_vjp(A.conj().T, beta, Ybar.conj().T)
        return Abar.conj().T, bb
    G = A.conj().T @ A
    lam, V = np.linalg.eigh(G)
    f, fb, F = svst_divided_differences(lam, beta)
    W = (V * f) @ V.conj().T
    Wbar = A.conj().T @ Ybar
    D = V.conj().T @ Wbar @ V
    K = V @ (F * (D + D.conj().T)) @ V.conj().T
    return Ybar @ W + A @ K, float(np.sum(fb * D.real.diagonal()))


def patch_svst_vjp(img: np.ndarray, beta: float, img_bar: np.ndarray, patch_size, stride_size):
    """Cotangent of ``patch_svst(img, β, ...)`` (src/recon.jl:251-256) with
    respect to img and β.  img2patches is a gather and patches2img a
    coverage-weighted sum, so their adjoints are a weighted gather and a
    scatter-add."""
    Nt, Nz, Ny, Nx = img.shape
    cnt = np.maximum(coverage_count((Nx, Ny, Nz), patch_size, stride_size), 1.0)
    P = img2patches(img, patch_size, stride_size)
    Pb = img2patches(img_bar / cnt[None], patch_size, stride_size)
    out = np.zeros_like(P)
    bsum = 0.0
    for ip in range(P.shape[0]):
        a, bb = svst_vjp(P[ip].T, beta, Pb[ip].T)
        out[ip] = a.T
        bsum += bb
    return patches2img(out, patch_size, stride_size, (Nx, Ny, Nz)) * cnt[None], bsum


def pogm_unrolled(prob: ReconProblem, niter: int, lambdas=None, L: float | None = None,
                  restart_cutoff: float = 0.0, bsig: float = 1.0, dtype=np.complex128):
    """Forward of the unrolled POGM from X0 = A'y (scripts/reconstruct.jl:209-226)
    with per-scale weights ``lambdas``.  Returns (X_niter, tape, restarts);
    tape[i] = (z_i, α, β_i, γ_i, ζ_i)."""
    Nx, Ny, Nz = prob.N
    Nt, Ns = prob.Nt, prob.Ns
    lam = list(prob.lambdas() if lambdas is None else lambdas)
    L = prob.lipschitz() if L is None else L
    smaps, y, idx, w = prob.smaps.astype(dtype), prob.y.astype(dtype), prob.idx, prob.workers
    x = np.zeros((Ns, Nt, Nz, Ny, Nx), dtype=dtype)
    x[0] = sense_adjoint(y, smaps, idx, w)
    u_old = x.copy()
    alpha = 1.0 / L
    t, sig = 1.0, 1.0
    gold = np.zeros_like(x)
    tape, restarts = [], [False]
    for it in range(1, niter + 1):
        g = sense_adjoint(sense_forward(x.sum(axis=0), smaps, idx, w) - y, smaps, idx, w)
        G = np.broadcast_to(g[None], x.shape)
        u = x - alpha * G
        tnew = 0.5 * (1 + math.sqrt(1 + (8 if it == niter else 4) * t * t))
        beta = (t - 1) / tnew
        gamma = sig * t / tnew
        z = u + beta * (u - u_old) + gamma * (u - x)
        zeta = alpha * (1 + beta + gamma)
        xn = np.empty_like(z)
        for k in range(Ns):
            xn[k] = patch_svst(z[k], zeta * lam[k], prob.patch_sizes[k], prob.strides[k])
        tape.append((z, alpha, beta, gamma, zeta))
        rs = _gr_restart(G, u - u_old, restart_cutoff)
        if rs:
            tnew, sig = 1.0, 1.0
        elif float(np.sum(np.real(G * gold), dtype=np.float64)) < 0:
            sig = bsig * sig
        restarts.append(bool(rs))
        gold = np.array(G)
        u_old, x, t = u, xn, tnew
    return x, tape, restarts


def unrolled_loss(X: np.ndarray, X_true: np.ndarray) -> float:
    """½ ‖Σ_k X_k − X_true‖² (FP64 sum)."""
    r = X.sum(axis=0).astype(np.complex128) - X_true
    return 0.5 * float(np.vdot(r, r).real)


def pogm_unrolled_grad(prob: ReconProblem, niter: int, X_true: np.ndarray, lambdas=None,
                       L: float | None = None, restart_cutoff: float = 0.0, bsig: float = 1.0):
    """loss and ∂loss/∂log λ_k of the unrolled POGM by reverse accumulation
    through the stored z_i (the eigen-decompositions are recomputed)."""
    lam = list(prob.lambdas() if lambdas is None else lambdas)
    X, tape, restarts = pogm_unrolled(prob, niter, lam, L, restart_cutoff, bsig)
    smaps, idx, w = prob.smaps.astype(np.complex128), prob.idx, prob.workers
    Ns = prob.Ns
    r = X.sum(axis=0) - X_true
    loss = 0.5 * float(np.vdot(r, r).real)
    xbar = np.broadcast_to(r[None], X.shape).copy()
    ubar = np.zeros_like(X)
    grad = np.zeros(Ns)
    for z, alpha, beta, gamma, zeta in reversed(tape):
        zbar = np.empty_like(z)
        for k in range(Ns):
            thr = zeta * lam[k]
            zbar[k], bb = patch_svst_vjp(z[k], thr, xbar[k], prob.patch_sizes[k], prob.strides[k])
            grad[k] += thr * bb
        wv = ubar + (1 + beta + gamma) * zbar
        hw = normal_op(wv.sum(axis=0), smaps, idx, w)
        xbar = wv - alpha * hw[None] - gamma * zbar
        ubar = -beta * zbar
    return loss, grad, X, restarts


# ---------------------------------------------------------------------------
# Setup of run_recon — scripts/reconstruct.jl:86-147, src/recon.jl:310-321
# ---------------------------------------------------------------------------
class SetupError(ValueError):
    """The reference's @assert failures of scripts/reconstruct.jl:113-118."""


def sos_normalize_maps(smaps_raw: np.ndarray) -> np.ndarray:
    """scripts/reconstruct.jl:89: ``S ./ (sqrt.(sum(abs2.(S); dims=4)) .+ eps(Float32))``
    in Float32, coils summed in order.  smaps_raw (Nc, Nz, Ny, Nx) complex64."""
    S = smaps_raw.astype(np.complex64)
    acc = np.zeros(S.shape[1:], dtype=np.float32)
    for c in range(S.shape[0]):
        acc = acc + (S[c].real * S[c].real + S[c].imag * S[c].imag)
    den = np.sqrt(acc) + np.finfo(np.float32).eps
    out = np.empty_like(S)
    out.real = S.real / den
    out.imag = S.imag / den
    return out


def sense_comb(ksp: np.ndarray, smaps: np.ndarray) -> np.ndarray:
    """src/recon.jl:310-321 on the zero-filled k-space ksp (Nt, Nc, Nz, Ny, Nx):
    Σ_c conj(S_c)·fftshift(ifft(ifftshift(ksp_c))) / (Σ_c |S_c|² + eps()),
    the denominator and the division in Float64, the image stored as
    ComplexF32."""
    den = np.sum(np.abs(smaps.astype(np.complex128)) ** 2, axis=0) + np.finfo(np.float64).eps
    img = np.empty((ksp.shape[0],) + ksp.shape[2:], dtype=np.complex64)
    for t in range(ksp.shape[0]):
        mc = sfft.fftshift(sfft.ifftn(sfft.ifftshift(ksp[t].astype(np.complex128), axes=SPATIAL_AXES),
                                      axes=SPATIAL_AXES), axes=SPATIAL_AXES)
        num = np.sum(np.conj(smaps.astype(np.complex128)) * mc, axis=0)
        img[t] = (num / den).astype(np.complex64)
    return img


def quantile_type7(v: np.ndarray, p: float) -> float:
    """Statistics.quantile (Hyndman–Fan type 7) as Julia evaluates it for a
    Float32 vector: a + γ·(b − a) with (b − a) in Float32 and the rest in
    Float64."""
    v = np.sort(np.asarray(v, dtype=np.float32).ravel())
    n = v.size
    h = (n - 1) * p
    j = int(math.floor(h))
    g = h - j
    a = v[j]
    b = v[min(j + 1, n - 1)]
    return float(a) + g * float(np.float32(b - a))


def prepare_kspace(ksp: np.ndarray, smaps_raw: np.ndarray):
    """scripts/reconstruct.jl:86-147 from the zero-filled k-space ksp
    (Nt, Nc, Nz, Ny, Nx) and raw coil maps (Nc, Nz, Ny, Nx).  Returns
    (smaps, y (Nt, Nc, K), idx (Nt, K) 0-based, scale_factor)."""
    smaps = sos_normalize_maps(smaps_raw)
    img0 = sense_comb(ksp, smaps)
    mags = np.abs(img0.astype(np.complex128)).astype(np.float32)
    scale = quantile_type7(mags, 0.99)
    div = max(scale, float(np.finfo(np.float32).eps))
    k = (ksp.astype(np.complex128) / div).astype(np.complex64)
    Nt, Nc = k.shape[:2]
    flat = k.reshape(Nt, Nc, -1)
    omega = flat[:, 0] != 0
    for c in range(1, Nc):
        if not np.array_equal(omega, flat[:, c] != 0):
            raise SetupError(f"Coil {c + 1} has a different sampling pattern")
    counts = omega.sum(axis=1)
    for t in range(1, Nt):
        if counts[t] != counts[t - 1]:
            raise SetupError(f"Frame {t + 1} has a different sample count")
    idx = np.stack([np.flatnonzero(omega[t]) for t in range(Nt)]).astype(np.int32)
    y = np.stack([flat[t][:, idx[t]] for t in range(Nt)])
    return smaps, y, idx, scale
