"""POGM over several GPUs: one rank per GPU, frames sharded for the SENSE
normal operator, z-slabs sharded for the patch SVST.

The reference runs on one device (scripts/reconstruct.jl:142 builds one
block-diagonal operator over all frames; src/sense_gpu.jl:124 takes one SVD
of the global patch).  One POGM iteration does not shard in a single layout:
the SENSE operator is independent per frame, patch SVST needs every frame of
a patch.  So each rank r holds

- a context for its block of frames F_r (coil maps, its frames' samples, A'y
  and the POGM state): the normal operator, the u/z update and the restart
  sums are computed there, in frame layout (Ns, |F_r|, Nz, Ny, Nx);
- a context for its z-slab Z_r of the volume over all frames: the patch SVST,
  in slab layout (Ns, Nt, |Z_r|, Ny, Nx).

Per iteration: the rank-local half of the step (``mslr_pogm_step_local``),
one all-reduce of the four restart totals, the restart decision (identical on
every rank), an all-to-all of z from frames to slabs, the SVST of every
scale on the slab — the global patch's Gram matrix Pᴴ P is a sum over voxels,
so each rank forms its slab's partial Gram, one all-reduce of the Nt × Nt
Gram, and each rank rebuilds its own rows — and an all-to-all of x back to
frames.  Scales other than the global patch must tile the volume with patch
boundaries on the slab boundaries (no halo exchange).

Collectives go through ``torch.distributed``: NCCL on device tensors, or gloo
through host copies (the CPU tests, and several ranks sharing one GPU).
"""
from __future__ import annotations

import ctypes as C
import math

import torch
import torch.distributed as dist

from ._lib import check, lib
from .context import MSLRContext, _dev_c64, _stream_ptr, ong_lustig_lambdas


def split_range(n: int, parts: int, unit: int = 1):
    """[start, stop) of each of `parts` contiguous blocks of range(n), in
    whole multiples of `unit`, as even as possible (earlier blocks larger)."""
    if n % unit:
        raise ValueError(f"{n} is not a multiple of {unit}")
    units = n // unit
    if parts < 1 or parts > units:
        raise ValueError(f"cannot split {units} blocks of {unit} into {parts} non-empty parts")
    base, extra = divmod(units, parts)
    out, s = [], 0
    for r in range(parts):
        e = s + (base + (1 if r < extra else 0)) * unit
        out.append((s, e))
        s = e
    return out


def slab_unit(N, patch_sizes, strides) -> int:
    """z granularity of the slabs: every scale is either the global patch or a
    tiling (stride = size, dividing the volume) whose z size the slab
    boundaries must respect."""
    Nz = N[2]
    unit = 1
    for ps, ss in zip(patch_sizes, strides):
        ps = [min(p, n) for p, n in zip(ps, N)]
        if list(ps) == list(N):
            continue
        if list(ps) != list(ss) or any(n % p for n, p in zip(N, ps)):
            raise ValueError(f"scale {ps} stride {ss}: the sharded iteration needs the global patch "
                             "or non-overlapping patches that tile the volume")
        unit = unit * ps[2] // math.gcd(unit, ps[2])
    if Nz % unit:
        raise ValueError("the patch z sizes do not divide the volume")
    return unit


def _sum_over_ranks(t: torch.Tensor, group=None):
    """In-place sum over the ranks (host copy for backends without device
    tensors)."""
    backend = dist.get_backend(group)
    if backend == "nccl" or not t.is_cuda:
        dist.all_reduce(t if not t.is_complex() else torch.view_as_real(t), group=group)
        return t
    h = t.cpu()
    dist.all_reduce(h if not h.is_complex() else torch.view_as_real(h), group=group)
    t.copy_(h)
    return t


def _all_to_all(send, recv, group=None):
    """send[q] goes to rank q, recv[q] comes from rank q (contiguous complex64
    tensors); through host buffers unless the backend takes device tensors."""
    device = send[0].device
    on_host = dist.get_backend(group) != "nccl" and device.type == "cuda"
    flat_s = torch.cat([s.reshape(-1) for s in send])
    if on_host:
        flat_s = flat_s.cpu()
    flat_r = torch.empty(sum(r.numel() for r in recv), dtype=flat_s.dtype, device=flat_s.device)
    dist.all_to_all_single(torch.view_as_real(flat_r).view(-1), torch.view_as_real(flat_s).view(-1),
                           [2 * r.numel() for r in recv], [2 * s.numel() for s in send], group=group)
    o = 0
    for r in recv:
        r.copy_(flat_r[o:o + r.numel()].view(r.shape))
        o += r.numel()


def frames_to_slabs(Zf: torch.Tensor, frames, slabs, rank: int, out: torch.Tensor, group=None):
    """Zf (Ns, |F_rank|, Nz, Ny, Nx) → out (Ns, Nt, |Z_rank|, Ny, Nx)."""
    send = [Zf[:, :, z0:z1].contiguous() for z0, z1 in slabs]
    z0, z1 = slabs[rank]
    recv = [torch.empty((Zf.shape[0], t1 - t0, z1 - z0) + tuple(Zf.shape[3:]), dtype=Zf.dtype,
                        device=Zf.device) for t0, t1 in frames]
    _all_to_all(send, recv, group)
    for (t0, t1), r in zip(frames, recv):
        out[:, t0:t1].copy_(r)
    return out


def slabs_to_frames(Xs: torch.Tensor, frames, slabs, rank: int, out: torch.Tensor, group=None):
    """Xs (Ns, Nt, |Z_rank|, Ny, Nx) → out (Ns, |F_rank|, Nz, Ny, Nx)."""
    send = [Xs[:, t0:t1].contiguous() for t0, t1 in frames]
    t0, t1 = frames[rank]
    recv = [torch.empty((Xs.shape[0], t1 - t0, z1 - z0) + tuple(Xs.shape[3:]), dtype=Xs.dtype,
                        device=Xs.device) for z0, z1 in slabs]
    _all_to_all(send, recv, group)
    for (z0, z1), r in zip(slabs, recv):
        out[:, :, z0:z1].copy_(r)
    return out


class ShardedRecon:
    """run_recon's POGM (mom=:pogm, restart=:gr) with the frames and the
    volume sharded over the ranks of `group` (one rank per GPU).

    ``N``, ``Nc``, ``Nt``, ``K``, ``patch_sizes``, ``strides`` describe the
    whole problem, as for :class:`MSLRContext`.  ``frames[r]`` and
    ``slabs[r]`` are rank r's [start, stop) frames and z planes.
    """

    def __init__(self, N, Nc: int, Nt: int, K: int, patch_sizes, strides, form: str = "tuned",
                 group=None):
        self.group = group
        self.P = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.N = tuple(int(v) for v in N)
        self.Nt, self.Nc, self.K = int(Nt), int(Nc), int(K)
        self.patch_sizes = [list(map(int, p)) for p in patch_sizes]
        self.strides = [list(map(int, s)) for s in strides]
        self.Ns = len(self.patch_sizes)
        self.lambdas = ong_lustig_lambdas(self.N, self.Nt, self.patch_sizes)   # of the whole problem
        self.frames = split_range(self.Nt, self.P)
        self.slabs = split_range(self.N[2], self.P, slab_unit(self.N, self.patch_sizes, self.strides))
        t0, t1 = self.frames[self.rank]
        z0, z1 = self.slabs[self.rank]
        Nx, Ny, _ = self.N
        self.global_scale = [[min(p, n) for p, n in zip(ps, self.N)] == list(self.N)
                             for ps in self.patch_sizes]
        # the slab's scales: the global patch becomes the slab's one patch
        sp = [[Nx, Ny, z1 - z0] if g else ps for ps, g in zip(self.patch_sizes, self.global_scale)]
        ss = [[Nx, Ny, z1 - z0] if g else st for st, g in zip(self.strides, self.global_scale)]
        for k, g in enumerate(self.global_scale):
            if g and Nx * Ny * (z1 - z0) < self.Nt:
                raise ValueError("a slab of the global patch has fewer voxels than frames")
        self.fctx = MSLRContext(self.N, Nc, t1 - t0, K, self.patch_sizes, self.strides, form=form)
        self.sctx = MSLRContext((Nx, Ny, z1 - z0), 1, self.Nt, 1, sp, ss, form=form)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.Xf = torch.empty((self.Ns, t1 - t0) + self.fctx.img_shape[1:], dtype=torch.complex64,
                              device=dev)
        self.Zf = torch.empty_like(self.Xf)
        self.Zs = torch.empty((self.Ns,) + self.sctx.img_shape, dtype=torch.complex64, device=dev)
        self.Xs = torch.empty_like(self.Zs)
        self.sums = torch.zeros(4, dtype=torch.float64, device=dev)
        self.gram = torch.empty((self.Nt, self.Nt), dtype=torch.complex64, device=dev)
        self.restarts = None

    def close(self):
        self.fctx.close()
        self.sctx.close()

    def bind(self, smaps: torch.Tensor, y_local: torch.Tensor, idx_local: torch.Tensor, index_base: int = 0):
        """Coil maps (Nc, Nz, Ny, Nx) and this rank's frames of the samples
        (|F_rank|, Nc, K) and indices (|F_rank|, K), CUDA tensors."""
        self.fctx.bind(smaps, y_local, idx_local, index_base=index_base)

    def _prox(self, zeta: float, stream):
        st = _stream_ptr(stream)
        for k in range(self.Ns):
            beta = zeta * self.lambdas[k]
            if self.global_scale[k]:
                check(lib.mslr_patch_gram(self.sctx._h, k, self.Zs[k].data_ptr(), self.gram.data_ptr(), st),
                      self.sctx._h)
                _sum_over_ranks(self.gram, self.group)
                check(lib.mslr_patch_svst_gram(self.sctx._h, k, float(beta), self.gram.data_ptr(),
                                               self.Zs[k].data_ptr(), self.Xs[k].data_ptr(), st), self.sctx._h)
            else:
                self.sctx.patch_svst(k, beta, self.Zs[k], out=self.Xs[k], stream=stream)

    def run(self, niter: int, L: float, restart_cutoff: float = 0.0, bsig: float = 1.0, callback=None,
            stream=None):
        """niter iterations from X0 = A'y; this rank's frames of X end in
        ``self.Xf``.  ``callback(it, Xf)`` sees them after every iteration.
        Returns the restart flags (niter + 1, as run_recon's logger)."""
        st = _stream_ptr(stream)
        f = self.fctx
        f.init_x0(self.Xf, stream=stream)
        f.pogm_begin(self.Xf, niter, L, restart_cutoff, bsig, stream=stream)
        abgz = (C.c_double * 4)()
        for it in range(1, niter + 1):
            check(lib.mslr_pogm_step_local(f._h, self.Xf.data_ptr(), self.Zf.data_ptr(), self.sums.data_ptr(), st),
                  f._h)
            _sum_over_ranks(self.sums, self.group)
            check(lib.mslr_pogm_step_decide(f._h, self.sums.data_ptr(), st), f._h)
            check(lib.mslr_pogm_scalars(f._h, abgz, st), f._h)
            frames_to_slabs(self.Zf, self.frames, self.slabs, self.rank, self.Zs, self.group)
            self._prox(float(abgz[3]), stream)
            slabs_to_frames(self.Xs, self.frames, self.slabs, self.rank, self.Xf, self.group)
            if callback is not None:
                callback(it, self.Xf)
        self.restarts = f.pogm_restarts(stream=stream)
        self.sctx.sync(stream=stream)
        return self.restarts
