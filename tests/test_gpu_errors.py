"""Device-side error reporting: bounded waits that run out, on the GPU,
without faulting it.

The tcgen05 kernels' mbarrier waits give up after a settable number of polls
(``mslr_set_wait_limit``).  With the limit at 0 every such wait gives up at
once; the kernel then still waits (with the default count) for the MMAs it
already issued, writes its output tile as zeros, frees its tensor memory and
records the time-out in the caller's error word.  These tests check that the
entry points return ``MSLR_ERR_CUDA`` with a message naming the time-out, and
that the next call with the default limit matches the FP64 oracle again.
"""
import numpy as np
import pytest

from oracle import mslr_oracle as O

pytestmark = pytest.mark.gpu

DEFAULT_POLLS = 1 << 22


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def M():
    import mslr_recon_b200 as M
    return M


def _batch(m, n, batch, seed):
    rng = np.random.default_rng(seed)
    X = (rng.standard_normal((batch, m, n)) + 1j * rng.standard_normal((batch, m, n))).astype(np.complex64)
    betas = [0.9 * float(np.median(np.linalg.svd(X[b], compute_uv=False))) for b in range(batch)]
    return X, betas


def test_svst_batch_wait_timeout_reported_then_recovers(torch, M):
    from mslr_recon_b200._lib import MSLR_ERR_CUDA, MSLRError, check, lib
    m, n, batch = 216, 64, 4
    X, betas = _batch(m, n, batch, 5)
    cm = torch.from_numpy(np.ascontiguousarray(np.transpose(X, (0, 2, 1)))).cuda()
    check(lib.mslr_set_wait_limit(None, 0))
    try:
        with pytest.raises(MSLRError) as ei:
            M.svst_batch(cm, m, n, betas)
        assert ei.value.code == MSLR_ERR_CUDA
        assert "timed out" in str(ei.value)
    finally:
        check(lib.mslr_set_wait_limit(None, DEFAULT_POLLS))
    out = np.transpose(M.svst_batch(cm, m, n, betas).cpu().numpy(), (0, 2, 1))
    for b in range(batch):
        assert O.rel_err(out[b], O.svst(X[b].astype(np.complex128), betas[b])) < 1e-4


def _small(pb):
    return O.ReconProblem(smaps=pb["smaps"].astype(np.complex128), idx=pb["idx"],
                          y=pb["y"].astype(np.complex128), patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"], sigma1=1.0)


def test_context_wait_timeout_reported_then_recovers(torch, M, small_problem):
    """A POGM iteration of the tuned form with every tcgen05 wait cut short:
    mslr_pogm_step returns (it does not synchronise), the next synchronising
    call reports the time-out, and a fresh run with the default limit
    matches the oracle's trajectory."""
    from mslr_recon_b200._lib import MSLR_ERR_CUDA, MSLRError
    pb = small_problem
    Nt, Nc, K = pb["y"].shape
    niter = 3
    traj = []
    _, restarts, _, _ = O.run_recon_arrays(_small(pb), niter,
                                           iter_callback=lambda it, xk, r: traj.append(xk.copy()))
    with M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form="tuned") as ctx:
        ctx.bind(torch.from_numpy(pb["smaps"]).cuda(), torch.from_numpy(pb["y"]).cuda(),
                 torch.from_numpy(pb["idx"]).to(torch.int32).cuda())
        L = float(len(pb["patch_sizes"]))
        X = ctx.init_x0()
        ctx.set_wait_limit(0)
        ctx.pogm_begin(X, niter, L)
        ctx.pogm_step(X)
        with pytest.raises(MSLRError) as ei:
            ctx.sync()
        assert ei.value.code == MSLR_ERR_CUDA
        assert "timed out" in str(ei.value)
        ctx.sync()   # the error word was cleared by the call that reported it
        ctx.set_wait_limit(DEFAULT_POLLS)
        X = ctx.init_x0()
        ctx.pogm_begin(X, niter, L)
        for i in range(niter):
            ctx.pogm_step(X)
            assert O.rel_err(X.cpu().numpy(), traj[i]) < 1e-4
        assert ctx.pogm_restarts() == restarts


def test_pogm_run_costs_matches_oracle(torch, M, small_problem):
    """mslr_pogm_run_costs: the iterate, the restart flags and run_recon's
    logged dc/reg costs (X0 and every iteration) against the FP64 oracle."""
    pb = small_problem
    Nt, Nc, K = pb["y"].shape
    niter = 6
    Xo, restarts, dcs, regs = O.run_recon_arrays(_small(pb), niter, log_costs=True)
    with M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form="tuned") as ctx:
        ctx.bind(torch.from_numpy(pb["smaps"]).cuda(), torch.from_numpy(pb["y"]).cuda(),
                 torch.from_numpy(pb["idx"]).to(torch.int32).cuda())
        X = ctx.init_x0()
        r, dc, reg = ctx.pogm_run_costs(X, niter, float(len(pb["patch_sizes"])))
        assert O.rel_err(X.cpu().numpy(), Xo) < 1e-4
    assert r == restarts   # entry 0 is the logger's X0 call, as in the oracle
    assert len(dc) == len(reg) == niter + 1 == len(dcs) == len(regs)
    for a, b in zip(dc, dcs):
        assert a == pytest.approx(b, rel=1e-4)
    for a, b in zip(reg, regs):
        assert a == pytest.approx(b, rel=1e-4)
