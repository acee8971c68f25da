"""Known-answer tests that pin the CPU oracle (the reference ships no tests or
golden vectors, so the oracle is pinned by the mathematics instead)."""
import math

import numpy as np
import pytest

from oracle import mslr_oracle as O


def cn(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / math.sqrt(2)


# --- patch geometry: src/recon.jl:54-72 ------------------------------------------
@pytest.mark.parametrize("N,ps,ss,np_expect,nsteps", [
    ((32, 32, 24), (6, 6, 6), (6, 6, 6), 144, (5, 5, 3)),          # small workload
    ((90, 90, 60), (90, 90, 60), (90, 90, 60), 1, (0, 0, 0)),      # global scale
    ((90, 90, 60), (10, 10, 10), (10, 10, 10), 486, (8, 8, 5)),    # 10^3 scale
    ((90, 90, 60), (10, 10, 10), (5, 5, 5), 3179, (16, 16, 10)),   # half-overlapping
    ((90, 90, 60), (6, 6, 6), (3, 3, 3), 15979, (28, 28, 18)),
    ((48, 48, 32), (8, 8, 8), (8, 8, 8), 144, (5, 5, 3)),
])
def test_geometry_counts(N, ps, ss, np_expect, nsteps):
    g = O.patch_geometry(N, ps, ss)
    assert g.Np == np_expect
    assert g.nsteps == nsteps


def test_geometry_clamped_edges():
    # 32 = 5*6 + 2: the last start is clamped to N - ps = 26 (1-based 27)
    g = O.patch_geometry((32, 32, 24), (6, 6, 6), (6, 6, 6))
    assert g.starts[0] == (0, 6, 12, 18, 24, 26)
    assert g.starts[2] == (0, 6, 12, 18)
    # patch larger than the image is clamped to it
    g = O.patch_geometry((5, 7, 3), (8, 8, 8), (4, 4, 4))
    assert g.ps == (5, 7, 3) and g.Np == 1


def test_patch_order_x_fastest():
    g = O.patch_geometry((12, 8, 4), (4, 4, 4), (4, 4, 4))
    assert [g.patch_start(i) for i in range(4)] == [(0, 0, 0), (4, 0, 0), (8, 0, 0), (0, 4, 0)]


@pytest.mark.parametrize("ps,ss", [((4, 4, 4), (4, 4, 4)), ((4, 3, 5), (2, 3, 1)), ((6, 6, 6), (6, 6, 6)),
                                   ((5, 5, 5), (3, 4, 2))])
def test_extract_recombine_identity(ps, ss):
    """patches2img(img2patches(x)) == x whenever stride <= patch size."""
    rng = np.random.default_rng(1)
    img = cn(rng, 3, 9, 10, 13)
    P = O.img2patches(img, ps, ss)
    back = O.patches2img(P, ps, ss, (13, 10, 9))
    np.testing.assert_allclose(back, img, rtol=1e-12, atol=1e-12)


def test_recombine_gaps_are_zero():
    rng = np.random.default_rng(2)
    img = cn(rng, 2, 1, 1, 10)
    P = O.img2patches(img, (2, 1, 1), (4, 1, 1))   # covers x = 0,1,4,5,8,9 (last clamped to 8)
    back = O.patches2img(P, (2, 1, 1), (4, 1, 1), (10, 1, 1))
    cov = O.coverage_count((10, 1, 1), (2, 1, 1), (4, 1, 1))[0, 0]
    assert list(cov) == [1, 1, 0, 0, 1, 1, 0, 0, 1, 1]
    assert np.all(back[..., cov == 0] == 0)


# --- SVST: src/recon.jl:183-211 ----------------------------------------------------
def test_svst_known_spectrum():
    rng = np.random.default_rng(3)
    U, _ = np.linalg.qr(cn(rng, 40, 6))
    V, _ = np.linalg.qr(cn(rng, 12, 6))
    s = np.array([10.0, 7.0, 4.0, 2.5, 1.0, 0.2])
    X = (U * s) @ V.conj().T
    out = O.svst(X, 3.0)
    expect = (U * np.maximum(s - 3.0, 0)) @ V.conj().T
    np.testing.assert_allclose(out, expect, atol=1e-10)


def test_svst_zero_and_full_threshold():
    X = np.zeros((5, 4), complex)
    assert np.all(O.svst(X, 1.0) == 0)
    rng = np.random.default_rng(4)
    Y = cn(rng, 5, 4)
    assert np.all(O.svst(Y, 1e6) == 0)
    np.testing.assert_allclose(O.svst(Y, 0.0), Y, atol=1e-12)


def test_svst_single_row_is_group_soft_threshold():
    rng = np.random.default_rng(5)
    x = cn(rng, 1, 30)
    nrm = np.linalg.norm(x)
    out = O.svst(x, 0.5 * nrm)
    np.testing.assert_allclose(out, x * 0.5, atol=1e-12)


# --- SENSE: src/sense_gpu.jl:51-101 ---------------------------------------------------
def _tiny_sense(rng, N=(6, 5, 4), Nc=3, frac=0.4):
    Nx, Ny, Nz = N
    smaps = cn(rng, Nc, Nz, Ny, Nx)
    smaps /= np.sqrt(np.sum(np.abs(smaps) ** 2, axis=0))[None]
    nvox = Nx * Ny * Nz
    idx = np.sort(rng.choice(nvox, int(frac * nvox), replace=False))
    return smaps, idx


def test_sense_adjointness():
    rng = np.random.default_rng(6)
    smaps, idx = _tiny_sense(rng)
    x = cn(rng, 4, 5, 6)
    y = cn(rng, 3, idx.size)
    lhs = np.vdot(O.sense_forward_frame(x, smaps, idx), y)
    rhs = np.vdot(x, O.sense_adjoint_frame(y, smaps, idx))
    assert abs(lhs - rhs) < 1e-12 * max(1, abs(lhs))


def test_sense_fully_sampled_is_isometry():
    rng = np.random.default_rng(7)
    smaps, _ = _tiny_sense(rng)
    idx = np.arange(smaps[0].size)
    x = cn(rng, 4, 5, 6)
    np.testing.assert_allclose(O.sense_adjoint_frame(O.sense_forward_frame(x, smaps, idx), smaps, idx),
                               x, atol=1e-12)


def test_sense_centring_matches_definition():
    """y[k] = s Σ_j S x_j ω^{(j-c)(k-c)} with c = n//2 per axis (odd axis included)."""
    rng = np.random.default_rng(8)
    N = (4, 3, 2)
    smaps = np.ones((1, 2, 3, 4), complex)
    x = cn(rng, 2, 3, 4)
    idx = np.arange(24)
    y = O.sense_forward_frame(x, smaps, idx)[0].reshape(2, 3, 4)
    ref = np.zeros((2, 3, 4), complex)
    for kz in range(2):
        for ky in range(3):
            for kx in range(4):
                acc = 0
                for jz in range(2):
                    for jy in range(3):
                        for jx in range(4):
                            ph = ((jx - 2) * (kx - 2) / 4 + (jy - 1) * (ky - 1) / 3 + (jz - 1) * (kz - 1) / 2)
                            acc += x[jz, jy, jx] * np.exp(-2j * np.pi * ph)
                ref[kz, ky, kx] = acc / math.sqrt(24)
    np.testing.assert_allclose(y, ref, atol=1e-12)


# --- λ and POGM ---------------------------------------------------------------------
def test_ong_lustig_lambdas():
    lam = O.ong_lustig_lambdas((90, 90, 60), 300, [[90, 90, 60], [10, 10, 10]])
    assert lam[0] == pytest.approx(716.846, abs=1e-3)
    assert lam[1] == pytest.approx(52.391, abs=1e-3)
    lam3 = O.ong_lustig_lambdas((90, 90, 60), 387, [[90, 90, 60], [10, 10, 10], [6, 6, 6]])
    assert lam3 == pytest.approx([719.250, 54.780, 37.988], abs=1e-3)
    assert O.ong_lustig_lambdas((32, 32, 24), 64, [[6, 6, 6]])[0] == pytest.approx(25.679, abs=1e-3)


def test_pogm_alias_recurrence():
    """With an in-place prox, the oracle's POGM equals the aliased recurrence
    written out by hand (no (xold - zold) term, Fgrad = fgrad, y = u)."""
    rng = np.random.default_rng(9)
    Q = rng.standard_normal((8, 8))
    H = Q @ Q.T / 8 + np.eye(8)
    b = rng.standard_normal(8)
    L = float(np.linalg.eigvalsh(H).max())

    def grad(x):
        return H @ x - b

    def prox(z, c):
        z[...] = np.sign(z) * np.maximum(np.abs(z) - 0.1 * c, 0)
        return z

    niter = 12
    x_or, _ = O.pogm_mod(np.zeros(8), lambda x: 0.0, grad, L, niter=niter, g_prox=prox)
    # hand recurrence
    x = np.zeros(8)
    u_old = x.copy()
    t = 1.0
    alpha = 1 / L
    for it in range(1, niter + 1):
        g = grad(x)
        u = x - alpha * g
        tn = 0.5 * (1 + math.sqrt(1 + (8 if it == niter else 4) * t * t))
        beta, gamma = (t - 1) / tn, t / tn
        z = u + beta * (u - u_old) + gamma * (u - x)
        xn = prox(z.copy(), alpha * (1 + beta + gamma))
        if np.sum(-g * (u - u_old)) <= 0:
            tn = 1.0
        u_old, x, t = u, xn, tn
    np.testing.assert_allclose(x_or, x, rtol=1e-12, atol=1e-12)


def test_power_iteration_matches_svd():
    rng = np.random.default_rng(10)
    A = rng.standard_normal((7, 5))
    _, s1 = O.poweriter_mod(lambda v: A @ v, lambda v: A.T @ v, np.ones(5), niter=500, tol=1e-12)
    assert s1 == pytest.approx(np.linalg.svd(A, compute_uv=False)[0], rel=1e-8)


def test_golden_fixtures_reproduce():
    """The committed fixtures (tests/golden/make_golden.py) are reproduced
    by the oracle."""
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "golden_small.npz")
    if not os.path.exists(path):
        pytest.skip("golden fixtures not generated")
    from tests.golden.make_golden import compute
    fresh = compute()
    ref = np.load(path)
    for k in ref.files:
        np.testing.assert_allclose(fresh[k], ref[k], rtol=1e-9, atol=1e-9, err_msg=k)


@pytest.mark.parametrize("case", ["small", "overlap", "bsig"])
def test_large_runner_is_run_recon_arrays(synth, case):
    """The full-size runner (threads over frames, patches and update chunks,
    shifts moved onto the coil maps, in-place recurrence with the aliasing
    resolved) gives run_recon_arrays' iterates and restart flags: the runner
    the full-size parity tests use is the same oracle."""
    import dataclasses
    kw = {}
    if case == "small":
        cfg = dataclasses.replace(synth.CONFIGS["small"], Nt=16)
    elif case == "overlap":   # a global patch, half-overlapping and clamped edge patches
        cfg = dataclasses.replace(synth.CONFIGS["small"], N=(14, 12, 10), Nt=10, Nc=4,
                                  patch_sizes=[[14, 12, 10], [4, 4, 4], [3, 3, 3]],
                                  strides=[[14, 12, 10], [2, 2, 2], [3, 3, 3]])
    else:                     # the σ decrease of pogm_mod (bsig < 1), no restarts
        cfg = dataclasses.replace(synth.CONFIGS["small"], N=(12, 10, 8), Nt=12, Nc=3,
                                  patch_sizes=[[12, 10, 8], [4, 5, 4]], strides=[[12, 10, 8], [4, 5, 4]])
        kw = {"bsig": 0.5, "restart_cutoff": -0.3}
    pb = synth.make_problem(cfg)
    prob = O.ReconProblem(smaps=pb["smaps"].astype(np.complex128), idx=pb["idx"],
                          y=pb["y"].astype(np.complex128), patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"], sigma1=0.7, workers=1)
    niter = 8
    ref = []
    _, r_ref, _, _ = O.run_recon_arrays(prob, niter, iter_callback=lambda it, xk, r: ref.append(xk.copy()),
                                        **kw)
    got = []
    _, r_got = O.run_recon_large(prob, niter, iter_callback=lambda it, xk, r: got.append(xk.copy()),
                                 threads=3, chunk=1000, **kw)
    assert r_got == r_ref
    for a, b in zip(got, ref):
        assert O.rel_err(a, b) < 1e-12
        assert O.rel_err_chunked(a, b, chunk=777) == pytest.approx(O.rel_err(a, b), rel=1e-9, abs=1e-300)


def test_weighted_nucnorm_matches_definition():
    """patch_nucnorm(P, λs) (src/recon.jl:154-166): the weighted sum of the
    patches' nuclear norms over Np; a zero patch adds nothing."""
    rng = np.random.default_rng(12)
    P = rng.standard_normal((4, 6, 5)) + 1j * rng.standard_normal((4, 6, 5))
    P[2] = 0
    lams = np.array([0.5, 2.0, 7.0, 1.5])
    want = sum(lams[i] * np.linalg.svd(P[i], compute_uv=False).sum() for i in (0, 1, 3)) / 4
    assert O.patch_nucnorm_weighted(P, lams) == pytest.approx(want, rel=1e-12)
    assert O.patch_nucnorm(P) == pytest.approx(sum(np.linalg.svd(P[i], compute_uv=False).sum() for i in range(4)))
