"""The unrolled-POGM gradient through the C ABI (mslr_pogm_grad): against the
FP64 oracle's reverse accumulation on small problems (overlapping and
partitioning patch grids, tall and wide patches, both forms), and at the
differentiation workload — 48×48×32, 12 coils, Nt = 128, scales [48,48,32]
and [8,8,8], 10 iterations — against the FP64 oracle's gradient and FP64
central finite differences (h = 1e-3 in log λ_k), to 1e-3.  (Finite
differences of the FP32 forward itself are limited by its rounding at about
1e-2 for this h, so the differences are taken in FP64.)"""
import importlib.util
import os
import sys

import numpy as np
import pytest

from oracle import mslr_oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def M():
    import mslr_recon_b200 as M
    return M


@pytest.fixture(scope="module")
def S():
    spec = importlib.util.spec_from_file_location("mslr_synth_grad",
                                                  os.path.join(os.path.dirname(HERE), "mslr-recon_b200",
                                                               "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    elif t.is_complex():
        t = t.to(torch.complex64)
    return t.cuda()


def problem(S, N, Nc, Nt, ps, ss, seed, rank=2, frac=0.4, centre=2):
    cfg = S.SynthConfig(N=N, Nc=Nc, Nt=Nt, rank=rank, frac=frac, centre=centre, seed=seed,
                        patch_sizes=ps, strides=ss)
    return S.make_problem(cfg)


def context(torch, M, pb, form):
    Nt, Nc, K = pb["y"].shape
    ctx = M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form=form)
    ctx.bind(dev(torch, pb["smaps"]), dev(torch, pb["y"]), dev(torch, pb["idx"], torch.int32))
    return ctx


@pytest.mark.parametrize("form", ["plain", "tuned"])
@pytest.mark.parametrize("case", ["overlap", "partition", "medium", "nt128"])
def test_gradient_vs_fp64_oracle(torch, M, S, form, case):
    if case == "overlap":
        pb = problem(S, (8, 6, 4), 3, 6, [[8, 6, 4], [4, 3, 2]], [[8, 6, 4], [2, 3, 2]], 100)
    elif case == "partition":
        pb = problem(S, (8, 6, 4), 3, 6, [[8, 6, 4], [4, 3, 2]], [[8, 6, 4], [4, 3, 2]], 101)
    elif case == "medium":
        pb = problem(S, (16, 16, 8), 4, 16, [[16, 16, 8], [4, 4, 4]], [[16, 16, 8], [4, 4, 4]], 102,
                     rank=3, frac=0.3, centre=4)
    else:   # Gram side 128 (tall patches, eigenvectors in global memory) and 64 (wide patches)
        pb = problem(S, (16, 16, 8), 4, 128, [[16, 16, 8], [8, 8, 8], [4, 4, 4]],
                     [[16, 16, 8], [8, 8, 8], [4, 4, 4]], 103, rank=4, frac=0.3, centre=4)
    prob = O.ReconProblem(smaps=pb["smaps"].astype(np.complex128), idx=pb["idx"],
                          y=pb["y"].astype(np.complex128), patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"])
    lam = [0.3 * v for v in prob.lambdas()]
    Xt = pb["x_true"].astype(np.complex128)
    niter = 5
    L = float(prob.Ns)
    loss_o, grad_o, X_o, restarts_o = O.pogm_unrolled_grad(prob, niter, Xt, lam, L)
    with context(torch, M, pb, form) as ctx:
        ctx.set_lambdas(lam)
        loss, grad, X, restarts = ctx.pogm_grad(dev(torch, pb["x_true"]), niter, L)
    assert restarts == restarts_o
    assert O.rel_err(X.cpu().numpy(), X_o) < 1e-4
    assert loss == pytest.approx(loss_o, rel=1e-4)
    scale = max(abs(g) for g in grad_o)
    assert scale > 0
    for g, go in zip(grad, grad_o):
        assert abs(g - go) <= 1e-3 * scale, (grad, grad_o)


GOLD = os.path.join(HERE, "golden", "grad_diff.npz")


@pytest.mark.parametrize("form", ["plain", "tuned"])
def test_gradient_diff_workload_vs_fp64(torch, M, S, form):
    """At the differentiation workload the gradient agrees to 1e-3 with the
    FP64 oracle's reverse accumulation and with FP64 central finite
    differences (h = 1e-3) of the oracle's forward, both precomputed by
    tests/golden/make_grad_golden.py on the same seeded inputs."""
    gold = dict(np.load(GOLD))
    pb = S.make_problem(S.CONFIGS["diff"])   # scipy FFTs: the fixture's inputs
    niter, L = int(gold["niter"]), float(gold["L"])
    with context(torch, M, pb, form) as ctx:
        np.testing.assert_allclose(ctx.lambdas, gold["lambdas"], rtol=1e-12)
        loss, grad, X, restarts = ctx.pogm_grad(dev(torch, pb["x_true"]), niter, L)
    assert restarts == [bool(v) for v in gold["restarts"]]
    assert loss == pytest.approx(float(gold["loss"]), rel=1e-4)
    for g, go, fd in zip(grad, gold["grad"], gold["fd"]):
        assert g == pytest.approx(float(go), rel=1e-3), (grad, gold["grad"])
        assert g == pytest.approx(float(fd), rel=1e-3), (grad, gold["fd"])


def test_split_gram_with_several_large_patches(torch, M):
    """Scales with a few large patches (here 4 patches of 16³ voxels, Nt = 40)
    take the unsplit Gram: the context's patch SVST matches the oracle."""
    rng = np.random.default_rng(21)
    N, Nt, Nc, K = (32, 32, 16), 40, 2, 100
    nvox = N[0] * N[1] * N[2]
    smaps = (rng.standard_normal((Nc, N[2], N[1], N[0])) + 0j).astype(np.complex64)
    idx = np.stack([np.sort(rng.choice(nvox, K, replace=False)) for _ in range(Nt)]).astype(np.int32)
    y = (rng.standard_normal((Nt, Nc, K)) + 1j * rng.standard_normal((Nt, Nc, K))).astype(np.complex64)
    U = rng.standard_normal((nvox, 3)) + 1j * rng.standard_normal((nvox, 3))
    V = rng.standard_normal((Nt, 3)) + 1j * rng.standard_normal((Nt, 3))
    img = ((V @ U.T) + 0.1 * (rng.standard_normal((Nt, nvox)) + 1j * rng.standard_normal((Nt, nvox))))
    img = img.reshape(Nt, N[2], N[1], N[0]).astype(np.complex64)
    ps = [16, 16, 16]
    with M.MSLRContext(N, Nc, Nt, K, [ps], [ps], form="tuned") as ctx:
        ctx.bind(dev(torch, smaps), dev(torch, y), dev(torch, idx, torch.int32))
        s = np.linalg.svd(O.img2patches(img.astype(np.complex128), ps, ps)[0].T, compute_uv=False)
        beta = float(0.5 * (s[3] + s[4]))
        out = ctx.patch_svst(0, beta, dev(torch, img)).cpu().numpy()
    ref = O.patch_svst(img.astype(np.complex128), beta, ps, ps)
    assert O.rel_err(out, ref) < 1e-4
