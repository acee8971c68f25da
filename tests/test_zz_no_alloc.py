"""The allocation-free batched SVST entry point.

Some callers of this library cannot call cudaMalloc: a host framework whose
memory pool owns the device (Julia's CUDA.jl, PyTorch's caching allocator)
must not have a library allocate behind the pool, and a real-time pipeline
may run on a fixed memory plan.  ``mslr_svst_batch_noalloc`` serves them by
using a fixed 16 MiB device array inside the library as its scratch.  This
test calls it through the C ABI twice in a row and compares each result with
the workspace-taking ``mslr_svst_batch`` on the same input, within the
tolerance the other SVST tests use, and with the FP64 oracle's SVST.  It
also checks that a bounded wait cut short (``mslr_set_wait_limit``) makes
the call fail instead of returning a partial result.  It lives in its own file, collected
last, and passes both alone in a fresh process and after the other tests.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import mslr_oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "mslr-recon_b200", "libmslr.so")


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_noalloc_matches_workspace_entry_point():
    import torch
    lib = C.CDLL(LIB)
    P, I32, D = C.c_void_p, C.c_int32, C.c_double
    lib.mslr_svst_batch_noalloc.argtypes = [I32, I32, I32, C.POINTER(D), P, P, P]
    lib.mslr_svst_batch.argtypes = [I32, I32, I32, C.POINTER(D), P, P, P, C.c_size_t, I32, P]
    lib.mslr_svst_batch_workspace.argtypes = [I32, I32, I32, C.POINTER(C.c_size_t)]
    lib.mslr_last_error.argtypes = [P]
    lib.mslr_last_error.restype = C.c_char_p

    m, n, batch = 216, 64, 12
    need = C.c_size_t()
    assert lib.mslr_svst_batch_workspace(m, n, batch, C.byref(need)) == 0
    assert need.value <= 16 * 1024 * 1024
    ws = torch.empty(need.value, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(2024)
    for call in range(2):
        X = (rng.standard_normal((batch, n, m)) + 1j * rng.standard_normal((batch, n, m))).astype(np.complex64)
        X[3] = 0   # a zero matrix must come back zero, as in the reference's zero-norm skip
        sv = [np.linalg.svd(X[b].T, compute_uv=False) for b in range(batch)]
        betas = (D * batch)(*[0.8 * float(np.median(s)) + call for s in sv])
        x_d = torch.from_numpy(X).cuda()
        out_na = torch.empty_like(x_d)
        out_ws = torch.empty_like(x_d)
        rc = lib.mslr_svst_batch_noalloc(m, n, batch, betas, x_d.data_ptr(), out_na.data_ptr(), stream)
        assert rc == 0, lib.mslr_last_error(None)
        rc = lib.mslr_svst_batch(m, n, batch, betas, x_d.data_ptr(), out_ws.data_ptr(), ws.data_ptr(),
                                 need.value, 1, stream)
        assert rc == 0, lib.mslr_last_error(None)
        torch.cuda.synchronize()
        a, b = out_na.cpu().numpy(), out_ws.cpu().numpy()
        assert np.all(a[3] == 0)
        assert _rel(a, b) < 2e-5, (call, _rel(a, b))
        # and against the FP64 oracle (thin SVD, singular values soft-thresholded)
        for k in (0, batch - 1):
            ref = O.svst(X[k].T.astype(np.complex128), betas[k]).T
            assert _rel(a[k], ref) < 1e-4, (call, k, _rel(a[k], ref))

    # a bounded wait that runs out is reported, not returned as a result: the
    # call fails with MSLR_ERR_CUDA, and the next call is right again
    lib.mslr_set_wait_limit.argtypes = [P, C.c_int64]
    assert lib.mslr_set_wait_limit(None, 0) == 0
    try:
        rc = lib.mslr_svst_batch_noalloc(m, n, batch, betas, x_d.data_ptr(), out_na.data_ptr(), stream)
        assert rc == 2
        assert b"timed out" in lib.mslr_last_error(None)
    finally:
        assert lib.mslr_set_wait_limit(None, 1 << 22) == 0
    rc = lib.mslr_svst_batch_noalloc(m, n, batch, betas, x_d.data_ptr(), out_na.data_ptr(), stream)
    assert rc == 0, lib.mslr_last_error(None)
    assert _rel(out_na.cpu().numpy(), out_ws.cpu().numpy()) < 2e-5

    # a batch larger than the fixed scratch is refused with a clear message
    bet = (D * 64)(*([1.0] * 64))
    big = torch.zeros((64, 300, 300), dtype=torch.complex64, device="cuda")
    rc = lib.mslr_svst_batch_noalloc(300, 300, 64, bet, big.data_ptr(), big.data_ptr(), stream)
    assert rc == 1
    assert b"scratch" in lib.mslr_last_error(None)
