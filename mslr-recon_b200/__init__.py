"""mslr-recon_b200 — B200-native MSLR POGM hot path.

A drop-in for the per-iteration path of rextlfung/mslr-recon: the SENSE
normal operator, per-scale patch singular-value soft-thresholding and the
POGM momentum / gradient-restart update, as hand-written sm_100a CUDA
kernels behind the C ABI of ``include/mslr.h`` (``libmslr.so`` in this
directory).  This Python layer mirrors the reference's Julia call surface
for tests and benchmarks; Julia callers use ``julia/MSLRB200.jl``.
"""
from ._lib import MSLRError, lib  # noqa: F401  (loads libmslr.so; raises if absent)
from .context import MSLRContext, fp32_peak, ong_lustig_lambdas, sampling  # noqa: F401
from .recon import SVST, img2patches, patch_geometry, patches2img, patchSVST, svst_batch  # noqa: F401
from .reconstruct import run_recon, run_recon_files, run_recon_kspace, sos_normalize  # noqa: F401

__all__ = ["MSLRContext", "MSLRError", "SVST", "img2patches", "patches2img", "patchSVST",
           "patch_geometry", "svst_batch", "run_recon", "run_recon_files", "run_recon_kspace", "sos_normalize", "ong_lustig_lambdas", "sampling", "fp32_peak"]
