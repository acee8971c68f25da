"""Owner of one ``mslr_ctx``: the device state run_recon builds
(scripts/reconstruct.jl:133-214) for one acquisition and patch schedule.

Device arrays are ``torch`` CUDA tensors (torch is used only for device
memory and streams).  Layouts are the reference's column-major Julia arrays
read as C-order tensors with reversed axes: image (Nt, Nz, Ny, Nx), X
(Ns, Nt, Nz, Ny, Nx), coil maps (Nc, Nz, Ny, Nx), k-space (Nt, Nc, K),
indices (Nt, K).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from ._lib import FORM_PLAIN, FORM_TF32, FORM_TUNED, check, i32arr, lib

FORMS = {"plain": FORM_PLAIN, "tuned": FORM_TUNED, "tf32": FORM_TF32}


def _stream_ptr(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _dev_c64(t, shape, name):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != torch.complex64:
        raise TypeError(f"{name} must be complex64, got {t.dtype}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t


def ong_lustig_lambdas(N, Nt, patch_sizes):
    """scripts/reconstruct.jl:163-169 (unclamped patch sizes)."""
    nvox = int(np.prod(N))
    out = []
    for ps in patch_sizes:
        p = int(np.prod(ps))
        out.append(math.sqrt(p) + math.sqrt(Nt) + math.sqrt(math.log(nvox * Nt / max(p, Nt))))
    return out


def sampling(ksp: torch.Tensor, idx=None, y=None, stream=None) -> int:
    """Samples per frame K of the zero-filled k-space ksp (Nt, Nc, Nz, Ny, Nx)
    — Ω from coil 1 with the checks of scripts/reconstruct.jl:109-118
    (ValueError with the reference's message otherwise); with idx (Nt, K)
    int32 and y (Nt, Nc, K) given, also gathers them (:144-147)."""
    if ksp.dim() != 5 or ksp.dtype != torch.complex64 or not ksp.is_cuda or not ksp.is_contiguous():
        raise ValueError("ksp must be a contiguous complex64 CUDA tensor (Nt, Nc, Nz, Ny, Nx)")
    Nt, Nc, Nz, Ny, Nx = ksp.shape
    K = C.c_int64()
    cap = idx.shape[1] if idx is not None else 0
    check(lib.mslr_sampling(i32arr([Nx, Ny, Nz]), Nc, Nt, ksp.data_ptr(), C.byref(K),
                            idx.data_ptr() if idx is not None else None,
                            y.data_ptr() if y is not None else None, cap, _stream_ptr(stream)))
    return int(K.value)


def fp32_peak(stream=None) -> float:
    """Measured FP32 FMA throughput of the current device, TFLOP/s."""
    v = C.c_double()
    check(lib.mslr_fp32_peak(C.byref(v), _stream_ptr(stream)))
    return float(v.value)


class MSLRContext:
    """One reconstruction context.

    ``N`` = (Nx, Ny, Nz); ``patch_sizes`` / ``strides`` are lists of (x, y, z)
    triples, one per scale; ``form`` is "plain" (FP32 SIMT) or "tuned".
    """

    def __init__(self, N, Nc: int, Nt: int, K: int, patch_sizes, strides, form: str = "tuned"):
        if len(patch_sizes) != len(strides) or not patch_sizes:
            raise ValueError("patch_sizes and strides must be non-empty and of equal length")
        self.N = tuple(int(v) for v in N)
        self.Nc, self.Nt, self.K = int(Nc), int(Nt), int(K)
        self.patch_sizes = [list(map(int, p)) for p in patch_sizes]
        self.strides = [list(map(int, s)) for s in strides]
        self.Ns = len(patch_sizes)
        self.form = form
        self.lambdas = ong_lustig_lambdas(self.N, self.Nt, self.patch_sizes)
        torch.cuda.init()
        h = C.c_void_p()
        flat_p = [v for p in self.patch_sizes for v in p]
        flat_s = [v for s in self.strides for v in s]
        rc = lib.mslr_create(i32arr(self.N), self.Nc, self.Nt, self.K, self.Ns, i32arr(flat_p),
                             i32arr(flat_s), FORMS[form], C.byref(h))
        check(rc, None)
        self._h = h
        self.bound = False

    # -- lifetime ------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.mslr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, rc):
        check(rc, self._h)

    @property
    def img_shape(self):
        Nx, Ny, Nz = self.N
        return (self.Nt, Nz, Ny, Nx)

    @property
    def x_shape(self):
        return (self.Ns,) + self.img_shape

    def workspace_bytes(self) -> int:
        b = C.c_size_t()
        self._chk(lib.mslr_workspace_bytes(self._h, C.byref(b)))
        return int(b.value)

    # -- acquisition -----------------------------------------------------------
    def bind(self, smaps: torch.Tensor, y: torch.Tensor, idx: torch.Tensor, index_base: int = 0,
             stream=None):
        """smaps (Nc,Nz,Ny,Nx) c64, y (Nt,Nc,K) c64, idx (Nt,K) int32 — all CUDA."""
        Nx, Ny, Nz = self.N
        _dev_c64(smaps, (self.Nc, Nz, Ny, Nx), "smaps")
        _dev_c64(y, (self.Nt, self.Nc, self.K), "y")
        if idx.dtype != torch.int32 or tuple(idx.shape) != (self.Nt, self.K) or not idx.is_cuda:
            raise ValueError("idx must be a CUDA int32 tensor of shape (Nt, K)")
        self._chk(lib.mslr_bind(self._h, smaps.data_ptr(), y.data_ptr(),
                                C.c_void_p(idx.contiguous().data_ptr()), index_base,
                                _stream_ptr(stream)))
        self.bound = True

    # -- operators -------------------------------------------------------------
    def forward(self, x: torch.Tensor, stream=None) -> torch.Tensor:
        _dev_c64(x, self.img_shape, "x")
        y = torch.empty((self.Nt, self.Nc, self.K), dtype=torch.complex64, device=x.device)
        self._chk(lib.mslr_sense_forward(self._h, x.data_ptr(), y.data_ptr(), _stream_ptr(stream)))
        return y

    def adjoint(self, y: torch.Tensor, stream=None) -> torch.Tensor:
        _dev_c64(y, (self.Nt, self.Nc, self.K), "y")
        x = torch.empty(self.img_shape, dtype=torch.complex64, device=y.device)
        self._chk(lib.mslr_sense_adjoint(self._h, y.data_ptr(), x.data_ptr(), _stream_ptr(stream)))
        return x

    def normal(self, X: torch.Tensor, subtract_data: bool = True, out=None, stream=None):
        """g = A'(A Σ_k X_k − y)  (or A'A Σ_k X_k); X is (ns, Nt, Nz, Ny, Nx) or 4-D."""
        if X.dim() == 4:
            X = X.unsqueeze(0)
        ns = X.shape[0]
        _dev_c64(X, (ns,) + self.img_shape, "X")
        g = out if out is not None else torch.empty(self.img_shape, dtype=torch.complex64,
                                                    device=X.device)
        self._chk(lib.mslr_normal_op(self._h, X.data_ptr(), ns, g.data_ptr(),
                                     1 if subtract_data else 0, _stream_ptr(stream)))
        return g

    def cost(self, X: torch.Tensor, stream=None):
        """(dc_cost, reg_cost) of run_recon's logger (scripts/reconstruct.jl:176-194)
        for X (Ns, Nt, Nz, Ny, Nx); FP64."""
        import ctypes as C
        if X.dim() == 4:
            X = X.unsqueeze(0)
        ns = X.shape[0]
        _dev_c64(X, (ns,) + self.img_shape, "X")
        dc = C.c_double()
        reg = C.c_double()
        self._chk(lib.mslr_cost(self._h, X.data_ptr(), ns, C.byref(dc),
                                C.byref(reg) if ns == self.Ns else None, _stream_ptr(stream)))
        return float(dc.value), (float(reg.value) if ns == self.Ns else None)

    def set_graph(self, enable: bool):
        """Tuned form: replay the POGM iteration from a captured CUDA graph
        (default) or launch its kernels directly."""
        self._chk(lib.mslr_set_graph(self._h, 1 if enable else 0))

    def normal_profile(self, X: torch.Tensor, out=None, stream=None):
        """One normal operator with events around every kernel of every chunk:
        returns ({kernel: average ms per launch}, launches of each).  Kernels of
        the four-pass form: "pfwd" (forward plane pass), "zmask" (z pass with
        the mask), "padj" (inverse plane pass), "csum" (coil combine); of the
        three-kernel form: "zfwd", "xy", "zadj"."""
        import ctypes as C
        if X.dim() == 4:
            X = X.unsqueeze(0)
        ns = X.shape[0]
        _dev_c64(X, (ns,) + self.img_shape, "X")
        g = out if out is not None else torch.empty(self.img_shape, dtype=torch.complex64,
                                                    device=X.device)
        ms = (C.c_double * 4)()
        n = (C.c_int64 * 4)()
        self._chk(lib.mslr_normal_op_profile(self._h, X.data_ptr(), ns, g.data_ptr(),
                                             _stream_ptr(stream), ms, n))
        if n[3] > 0:
            return {"pfwd": ms[0], "zmask": ms[1], "padj": ms[2], "csum": ms[3]}, int(n[0])
        return {"zfwd": ms[0], "xy": ms[1], "zadj": ms[2]}, int(n[0])

    def patch_svst(self, scale: int, beta: float, img: torch.Tensor, out=None, stream=None):
        _dev_c64(img, self.img_shape, "img")
        o = out if out is not None else torch.empty_like(img)
        self._chk(lib.mslr_patch_svst(self._h, int(scale), float(beta), img.data_ptr(),
                                      o.data_ptr(), _stream_ptr(stream)))
        return o

    def patch_svst_lambdas(self, scale: int, lambdas, img: torch.Tensor, out=None, stream=None):
        """patchSVST(img, λs, ...) of scale `scale` with one threshold per patch
        (src/recon.jl:263-268)."""
        _dev_c64(img, self.img_shape, "img")
        lam = [float(v) for v in lambdas]
        o = out if out is not None else torch.empty_like(img)
        self._chk(lib.mslr_patch_svst_lambdas(self._h, int(scale), (C.c_double * len(lam))(*lam),
                                              img.data_ptr(), o.data_ptr(), _stream_ptr(stream)))
        return o

    def patch_nucnorm(self, scale: int, img: torch.Tensor, lambdas=None, stream=None) -> float:
        """patch_nucnorm of scale `scale`'s patches of img: Σ_p Σσ, or with
        per-patch weights Σ_p λ_p Σσ_p / Np (src/recon.jl:138-166)."""
        _dev_c64(img, self.img_shape, "img")
        lam = None if lambdas is None else (C.c_double * len(lambdas))(*[float(v) for v in lambdas])
        out = C.c_double()
        self._chk(lib.mslr_patch_nucnorm(self._h, int(scale), lam, img.data_ptr(), C.byref(out),
                                         _stream_ptr(stream)))
        return float(out.value)

    def init_x0(self, X=None, stream=None):
        X = X if X is not None else torch.empty(self.x_shape, dtype=torch.complex64, device="cuda")
        _dev_c64(X, self.x_shape, "X")
        self._chk(lib.mslr_init_x0(self._h, X.data_ptr(), _stream_ptr(stream)))
        return X

    # -- POGM --------------------------------------------------------------------
    def pogm_run(self, X: torch.Tensor, niter: int, L: float, restart_cutoff: float = 0.0,
                 bsig: float = 1.0, stream=None):
        _dev_c64(X, self.x_shape, "X")
        r = (C.c_uint8 * (niter + 1))()
        self._chk(lib.mslr_pogm_run(self._h, X.data_ptr(), int(niter), float(L),
                                    float(restart_cutoff), float(bsig), r, _stream_ptr(stream)))
        return [bool(v) for v in r]

    def pogm_run_costs(self, X: torch.Tensor, niter: int, L: float, restart_cutoff: float = 0.0,
                       bsig: float = 1.0, stream=None):
        """pogm_run that also returns run_recon's logged costs: (restarts,
        dc_costs, reg_costs), each of length niter+1 (X0, then after every
        iteration; scripts/reconstruct.jl:204-205, 228-230)."""
        _dev_c64(X, self.x_shape, "X")
        r = (C.c_uint8 * (niter + 1))()
        dc = (C.c_double * (niter + 1))()
        reg = (C.c_double * (niter + 1))()
        self._chk(lib.mslr_pogm_run_costs(self._h, X.data_ptr(), int(niter), float(L),
                                          float(restart_cutoff), float(bsig), r, dc, reg,
                                          _stream_ptr(stream)))
        self._niter = int(niter)
        return [bool(v) for v in r], [float(v) for v in dc], [float(v) for v in reg]

    MOMS = {"pgm": 0, "fpgm": 1, "pogm": 2}
    RESTARTS = {"none": 0, "gr": 1, "fr": 2}

    def pogm_run_options(self, X: torch.Tensor, niter: int, L: float, mom: str = "pogm",
                         restart: str = "gr", f_mu: float = 0.0, restart_cutoff: float = 0.0,
                         bsig: float = 1.0, stream=None):
        """pogm_mod with any of its options (src/mirt_mod.jl:74-188): ``mom``
        in ("pgm", "fpgm", "pogm"), ``restart`` in ("none", "gr", "fr"),
        ``f_mu`` >= 0.  X (x0 on entry) receives pogm_mod's result (x for
        :pogm, y for :pgm / :fpgm).  Returns the restart flags (niter + 1)."""
        _dev_c64(X, self.x_shape, "X")
        if mom not in self.MOMS:
            raise ValueError(f"mom={mom}")
        if restart not in self.RESTARTS:
            raise ValueError(f"restart={restart}")
        r = (C.c_uint8 * (niter + 1))()
        self._chk(lib.mslr_pogm_run_options(self._h, X.data_ptr(), int(niter), float(L), float(f_mu),
                                            self.MOMS[mom], self.RESTARTS[restart], float(restart_cutoff),
                                            float(bsig), r, _stream_ptr(stream)))
        self._niter = int(niter)
        return [bool(v) for v in r]

    def sync(self, stream=None):
        """Synchronise the stream and raise any device-side error the
        context's kernels recorded since the last check."""
        self._chk(lib.mslr_sync(self._h, _stream_ptr(stream)))

    def set_wait_limit(self, polls: int):
        """Polls of a tensor-core kernel's bounded wait before it gives up
        (default 2**22); small values exist to test the time-out path."""
        self._chk(lib.mslr_set_wait_limit(self._h, int(polls)))

    def pogm_begin(self, X, niter, L, restart_cutoff=0.0, bsig=1.0, stream=None):
        _dev_c64(X, self.x_shape, "X")
        self._niter = int(niter)
        self._chk(lib.mslr_pogm_begin(self._h, X.data_ptr(), int(niter), float(L),
                                      float(restart_cutoff), float(bsig), _stream_ptr(stream)))

    def pogm_step(self, X, stream=None):
        self._chk(lib.mslr_pogm_step(self._h, X.data_ptr(), _stream_ptr(stream)))

    def pogm_restarts(self, stream=None):
        r = (C.c_uint8 * (self._niter + 1))()
        self._chk(lib.mslr_pogm_restarts(self._h, r, _stream_ptr(stream)))
        return [bool(v) for v in r]

    def prepare(self, ksp: torch.Tensor, smaps_raw: torch.Tensor, stream=None):
        """scripts/reconstruct.jl:86-147 on the device from the zero-filled
        k-space ksp (Nt, Nc, Nz, Ny, Nx) and raw coil maps (Nc, Nz, Ny, Nx):
        SOS-normalised maps, Ω and its checks, the samples y / indices idx,
        the scale factor quantile(|sense_comb|, 0.99), y scaled; the context
        is bound.  Returns (smaps, y, idx, scale_factor)."""
        _dev_c64(ksp, (self.Nt, self.Nc) + self.img_shape[1:], "ksp")
        _dev_c64(smaps_raw, (self.Nc,) + self.img_shape[1:], "smaps_raw")
        dev = ksp.device
        smaps = torch.empty_like(smaps_raw)
        y = torch.empty((self.Nt, self.Nc, self.K), dtype=torch.complex64, device=dev)
        idx = torch.empty((self.Nt, self.K), dtype=torch.int32, device=dev)
        sf = C.c_double()
        self._chk(lib.mslr_prepare(self._h, ksp.data_ptr(), smaps_raw.data_ptr(), smaps.data_ptr(),
                                   y.data_ptr(), idx.data_ptr(), C.byref(sf), _stream_ptr(stream)))
        return smaps, y, idx, float(sf.value)

    def autotune(self, stream=None):
        """Time the free launch shapes on the bound context and keep the
        fastest; returns the tuning (see tuning())."""
        self._chk(lib.mslr_autotune(self._h, _stream_ptr(stream)))
        return self.tuning()

    def tuning(self):
        """{'coils_per_group', 'frames_per_chunk', 'gram_splits': [per scale, 0 = heuristic],
        'lanes', 'zmask_ctas_per_sm', 'zmask_warps', 'eig_threads': [per scale]}"""
        n = C.c_int32()
        vals = (C.c_int32 * 64)()
        self._chk(lib.mslr_get_tuning(self._h, vals, 64, C.byref(n)))
        v = list(vals[:n.value])
        ns = self.Ns
        return {"coils_per_group": v[0], "frames_per_chunk": v[1], "gram_splits": v[2:2 + ns],
                "lanes": v[2 + ns], "zmask_ctas_per_sm": v[3 + ns], "zmask_warps": v[4 + ns],
                "eig_threads": v[5 + ns:5 + 2 * ns]}

    def set_lambdas(self, lambdas):
        """Per-scale weights λ_k of g_prox (scripts/reconstruct.jl:164-169, 196-202)."""
        lam = [float(v) for v in lambdas]
        if len(lam) != self.Ns:
            raise ValueError(f"need {self.Ns} lambdas")
        self._chk(lib.mslr_set_lambdas(self._h, (C.c_double * self.Ns)(*lam)))
        self.lambdas = lam

    def pogm_grad(self, X_true: torch.Tensor, niter: int, L: float, restart_cutoff: float = 0.0,
                  bsig: float = 1.0, X=None, stream=None):
        """Unrolled POGM from X0 = A'y and its gradient: returns (loss,
        d loss/d log λ_k per scale, X_niter, restart flags) for
        loss = ½‖Σ_k X_k − X_true‖²; X_true is (Nt, Nz, Ny, Nx)."""
        _dev_c64(X_true, self.img_shape, "X_true")
        if X is None:
            X = torch.empty(self.x_shape, dtype=torch.complex64, device=X_true.device)
        _dev_c64(X, self.x_shape, "X")
        loss = C.c_double()
        grad = (C.c_double * self.Ns)()
        r = (C.c_uint8 * (niter + 1))()
        self._chk(lib.mslr_pogm_grad(self._h, X_true.data_ptr(), int(niter), float(L),
                                     float(restart_cutoff), float(bsig), X.data_ptr(), C.byref(loss),
                                     grad, r, _stream_ptr(stream)))
        return float(loss.value), [float(g) for g in grad], X, [bool(v) for v in r]

    def launch_count(self) -> int:
        n = C.c_uint64()
        self._chk(lib.mslr_launch_count(self._h, C.byref(n)))
        return int(n.value)

    def power_iter(self, niter: int = 200, tol: float = 1e-6, stream=None):
        s = C.c_double()
        it = C.c_int32()
        self._chk(lib.mslr_power_iter(self._h, int(niter), float(tol), C.byref(s), C.byref(it),
                                      _stream_ptr(stream)))
        return float(s.value), int(it.value)
