"""Precision sweep of the patch-SVST products (the benchmark definition's
precision study): the FP32 SIMT form (plain), the split-BF16 tensor-core form
(tuned) and the TF32 tensor-core form (tf32), each against the FP64 oracle —
batched SVST of low-rank-plus-noise patches, and the relative error of the
POGM iterate after every iteration of the small workload and of the
precision workload's decaying spectrum (1/k^1.5) at 90×90×60 with few frames."""
import numpy as np
import pytest

from oracle import mslr_oracle as O

pytestmark = pytest.mark.gpu

# per-iteration bound on X (the benchmark's bar) for the FP32 and split-BF16
# forms; the TF32 form (10-bit mantissa products, ~3e-4 per SVST) is
# reported against a looser bound, and its restart flags are not required to
# match: on the small workload a restart test sits close enough to its
# threshold (Σ Re(−g·Δu) ≈ 0) for TF32's error to decide it either way, after
# which the trajectory differs by a few 1e-3
ITER_TOL = {"plain": 1e-4, "tuned": 1e-4, "tf32": 5e-3}
SVST_TOL = {"plain": 2e-5, "tuned": 1e-4, "tf32": 2e-3}


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def M():
    import mslr_recon_b200 as M
    return M


def dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    elif t.is_complex():
        t = t.to(torch.complex64)
    return t.cuda()


@pytest.mark.parametrize("form", ["plain", "tuned", "tf32"])
@pytest.mark.parametrize("m,n,batch", [(1000, 300, 2), (216, 64, 5), (40, 12, 5)])
def test_svst_batch_precision(torch, M, m, n, batch, form):
    rng = np.random.default_rng(m * 7 + n)
    X = (rng.standard_normal((batch, m, n)) + 1j * rng.standard_normal((batch, m, n))).astype(np.complex64)
    for b in range(batch):
        U = rng.standard_normal((m, 4)) + 1j * rng.standard_normal((m, 4))
        V = rng.standard_normal((4, n)) + 1j * rng.standard_normal((4, n))
        X[b] += (3.0 * U @ V).astype(np.complex64)
    betas = [0.9 * float(np.median(np.linalg.svd(X[b], compute_uv=False))) for b in range(batch)]
    cm = np.ascontiguousarray(np.transpose(X, (0, 2, 1)))
    from mslr_recon_b200.context import FORMS
    out = np.transpose(M.svst_batch(dev(torch, cm), m, n, betas, form=FORMS[form]).cpu().numpy(), (0, 2, 1))
    errs = [O.rel_err(out[b], O.svst(X[b].astype(np.complex128), betas[b])) for b in range(batch)]
    print(f"svst {form} {m}x{n}: max rel err {max(errs):.2e}")
    assert max(errs) < SVST_TOL[form], errs


def _per_iteration_errors(torch, M, pb, form, niter, L):
    Nt, Nc, K = pb["y"].shape
    prob = O.ReconProblem(smaps=pb["smaps"].astype(np.complex128), idx=pb["idx"],
                          y=pb["y"].astype(np.complex128), patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"], sigma1=np.sqrt(L / len(pb["patch_sizes"])))
    traj = []
    _, restarts, _, _ = O.run_recon_arrays(prob, niter, iter_callback=lambda it, xk, r: traj.append(xk.copy()))
    with M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form=form) as ctx:
        ctx.bind(dev(torch, pb["smaps"]), dev(torch, pb["y"]), dev(torch, pb["idx"], torch.int32))
        X = ctx.init_x0()
        ctx.pogm_begin(X, niter, L)
        errs = []
        for i in range(niter):
            ctx.pogm_step(X)
            errs.append(O.rel_err(X.cpu().numpy(), traj[i]))
        same = ctx.pogm_restarts() == restarts
    return errs, same


@pytest.mark.parametrize("form", ["plain", "tuned", "tf32"])
def test_precision_sweep_small_workload(torch, M, small_problem, form):
    errs, same = _per_iteration_errors(torch, M, small_problem, form, small_problem["niters"], 1.0)
    print(f"small workload {form}: max per-iteration rel err {max(errs):.2e} (last {errs[-1]:.2e}); "
          f"restart flags {'identical' if same else 'differ'}; per iteration "
          + " ".join(f"{e:.1e}" for e in errs))
    assert max(errs) < ITER_TOL[form], errs
    assert same or form == "tf32"


@pytest.mark.parametrize("form", ["plain", "tuned", "tf32"])
def test_precision_sweep_decaying_spectrum(torch, M, synth, form):
    """The precision workload (90×90×60, 18 coils, two scales, singular
    values decaying as 1/k^1.5) with 8 frames and 5 iterations."""
    import dataclasses
    cfg = dataclasses.replace(synth.CONFIGS["precision"], Nt=8)
    pb = synth.make_problem(cfg, fft="torch")
    errs, same = _per_iteration_errors(torch, M, pb, form, 5, 2.0)
    print(f"precision workload (Nt=8) {form}: max per-iteration rel err {max(errs):.2e}")
    assert max(errs) < ITER_TOL[form], errs
    assert same
