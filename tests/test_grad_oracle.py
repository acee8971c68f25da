"""The FP64 oracle of the unrolled-POGM gradient (∂loss/∂log λ_k), pinned by
finite differences of its own forward: the patch-SVST backward (Gram /
Daleckii–Krein form), the unrolled recurrence against pogm_mod, and the whole
reverse accumulation."""
import math

import numpy as np
import pytest

from oracle import mslr_oracle as O


def cn(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / math.sqrt(2)


def tiny_problem(seed=0, overlap=True):
    import importlib.util
    import os
    import sys
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("mslr_synth_t", os.path.join(here, "mslr-recon_b200",
                                                                                "synth.py"))
    S = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = S
    spec.loader.exec_module(S)
    cfg = S.SynthConfig(N=(8, 6, 4), Nc=3, Nt=6, rank=2, frac=0.4, centre=2, seed=100 + seed,
                        patch_sizes=[[8, 6, 4], [4, 3, 2]],
                        strides=[[8, 6, 4], [2, 3, 2] if overlap else [4, 3, 2]])
    pb = S.make_problem(cfg)
    prob = O.ReconProblem(smaps=pb["smaps"], idx=pb["idx"], y=pb["y"], patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"])
    return prob, pb["x_true"].astype(np.complex128)


@pytest.mark.parametrize("shape", [(9, 5), (4, 7)])
def test_svst_vjp_matches_finite_differences(shape):
    rng = np.random.default_rng(3)
    A = cn(rng, *shape)
    s = np.linalg.svd(A, compute_uv=False)
    beta = float(0.5 * (s[1] + s[2]))   # between singular values: two above, the rest below
    C = cn(rng, *shape)
    dA = cn(rng, *shape)

    def ell(a, b):
        return float(np.real(np.vdot(C, O.svst(a, b))))

    Abar, bb = O.svst_vjp(A, beta, C)
    h = 1e-6
    fd = (ell(A + h * dA, beta) - ell(A - h * dA, beta)) / (2 * h)
    assert float(np.real(np.vdot(Abar, dA))) == pytest.approx(fd, rel=1e-6, abs=1e-9)
    fdb = (ell(A, beta + h) - ell(A, beta - h)) / (2 * h)
    assert bb == pytest.approx(fdb, rel=1e-6, abs=1e-9)


def test_patch_svst_vjp_overlapping_patches():
    rng = np.random.default_rng(4)
    img = cn(rng, 5, 4, 6, 8)
    ps, ss = (4, 3, 2), (2, 3, 2)
    P = O.img2patches(img, ps, ss)
    s1 = [np.linalg.svd(P[i].T, compute_uv=False)[1] for i in range(P.shape[0])]
    beta = float(np.median(s1)) * 1.013   # off every patch's singular values
    C = cn(rng, *img.shape)
    d = cn(rng, *img.shape)

    def ell(x, b):
        return float(np.real(np.vdot(C, O.patch_svst(x, b, ps, ss))))

    zbar, bb = O.patch_svst_vjp(img, beta, C, ps, ss)
    h = 1e-6
    fd = (ell(img + h * d, beta) - ell(img - h * d, beta)) / (2 * h)
    assert float(np.real(np.vdot(zbar, d))) == pytest.approx(fd, rel=1e-6)
    fdb = (ell(img, beta + h) - ell(img, beta - h)) / (2 * h)
    assert bb == pytest.approx(fdb, rel=1e-6)


def test_unrolled_forward_is_pogm_mod():
    prob, _ = tiny_problem()
    lam = [0.3 * v for v in prob.lambdas()]
    X, _, restarts = O.pogm_unrolled(prob, 6, lam)

    # run_recon_arrays with the same λ
    orig = O.ong_lustig_lambdas
    try:
        O.ong_lustig_lambdas = lambda N, Nt, ps: lam
        Xr, rr, _, _ = O.run_recon_arrays(prob, 6)
    finally:
        O.ong_lustig_lambdas = orig
    assert O.rel_err(X, Xr) < 1e-12
    assert restarts == rr


@pytest.mark.parametrize("overlap", [False, True])
def test_unrolled_gradient_matches_finite_differences(overlap):
    prob, X_true = tiny_problem(overlap=overlap)
    lam = np.array([0.3 * v for v in prob.lambdas()])
    niter = 5
    loss, grad, _, restarts = O.pogm_unrolled_grad(prob, niter, X_true, list(lam))
    h = 1e-5
    for k in range(prob.Ns):
        e = np.zeros_like(lam)
        e[k] = h
        Xp, _, rp = O.pogm_unrolled(prob, niter, list(lam * np.exp(e)))
        Xm, _, rm = O.pogm_unrolled(prob, niter, list(lam * np.exp(-e)))
        assert rp == restarts and rm == restarts
        fd = (O.unrolled_loss(Xp, X_true) - O.unrolled_loss(Xm, X_true)) / (2 * h)
        assert grad[k] == pytest.approx(fd, rel=1e-6, abs=1e-10 * abs(loss))
