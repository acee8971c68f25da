"""GPU parity tests: every kernel path through the C ABI against the CPU
oracle / the committed golden fixtures.

Tolerances: patch indexing and masks are integer work and must be bit-exact;
floating-point results must match the FP64 oracle to a relative Frobenius
error of 1e-4 (the bound stated for the POGM iterate), with tighter bounds
where single FP32 operations are involved.
"""
import os

import numpy as np
import pytest

from oracle import mslr_oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_small.npz")
PATCHES = [[8, 6, 4], [4, 3, 2], [3, 3, 3]]
STRIDES = [[8, 6, 4], [4, 3, 2], [2, 2, 2]]


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
def gold():
    return dict(np.load(GOLD))


def dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    elif t.is_complex():
        t = t.to(torch.complex64)
    return t.cuda()


def rel(a, b):
    return O.rel_err(a, b)


# --- patch operators: bit-exact indexing -------------------------------------
@pytest.mark.parametrize("k", [0, 1, 2])
def test_img2patches_bit_exact(torch, M, gold, k):
    x = gold["x"].astype(np.complex64)
    P = M.img2patches(dev(torch, x), PATCHES[k], STRIDES[k]).cpu().numpy()
    ref = O.img2patches(x, PATCHES[k], STRIDES[k])
    assert P.shape == ref.shape
    assert np.array_equal(P, ref)


@pytest.mark.parametrize("N,ps,ss", [((13, 7, 5), (4, 4, 4), (3, 2, 4)), ((10, 1, 1), (2, 1, 1), (4, 1, 1)),
                                     ((9, 9, 9), (3, 3, 3), (3, 3, 3)), ((11, 6, 4), (20, 3, 2), (5, 1, 1))])
def test_recombine_matches_reference_order(torch, M, N, ps, ss):
    rng = np.random.default_rng(11)
    Nt = 5
    g = O.patch_geometry(N, ps, ss)
    P = (rng.standard_normal((g.Np, Nt, g.p)) + 1j * rng.standard_normal((g.Np, Nt, g.p))).astype(np.complex64)
    out = M.patches2img(dev(torch, P), ps, ss, N).cpu().numpy()
    ref = O.patches2img(P, ps, ss, N)   # float32 sums in ascending ip, same as the kernel
    np.testing.assert_array_equal(out, ref)


# --- SVST ------------------------------------------------------------------------
SVST_TOL = {"plain": 2e-5, "tuned": 1e-4}   # FP32 SIMT; split-precision BF16x3 tensor cores
NORMAL_TOL = {"plain": 1e-5, "tuned": 1e-5, "tuned-tc": 5e-5}   # FP32 FFTs; split-BF16 tensor-core plane DFTs


@pytest.mark.parametrize("form", ["plain", "tuned"])
@pytest.mark.parametrize("m,n,batch", [(40, 12, 5), (12, 40, 5), (216, 64, 7), (64, 216, 3), (1000, 300, 2),
                                       (1, 30, 4), (30, 1, 4), (150, 100, 3), (500, 384, 3), (63, 80, 3)])
def test_svst_batch_vs_oracle(torch, M, m, n, batch, form):
    rng = np.random.default_rng(m * 1000 + n)
    X = (rng.standard_normal((batch, m, n)) + 1j * rng.standard_normal((batch, m, n))).astype(np.complex64)
    # low-rank + noise so that thresholds land inside the spectrum
    r = min(4, m, n)
    for b in range(batch):
        U = rng.standard_normal((m, r)) + 1j * rng.standard_normal((m, r))
        V = rng.standard_normal((r, n)) + 1j * rng.standard_normal((r, n))
        X[b] += (3.0 * U @ V).astype(np.complex64)
    sv = [np.linalg.svd(X[b], compute_uv=False) for b in range(batch)]
    betas = [0.9 * float(np.median(s)) for s in sv]
    betas[0] = 0.0
    if batch > 2:
        X[2] = 0
        betas[2] = 1.0
    cm = np.ascontiguousarray(np.transpose(X, (0, 2, 1)))   # column-major storage
    from mslr_recon_b200.context import FORMS
    out = M.svst_batch(dev(torch, cm), m, n, betas, form=FORMS[form]).cpu().numpy()
    out = np.transpose(out, (0, 2, 1))
    for b in range(batch):
        ref = O.svst(X[b].astype(np.complex128), betas[b])
        if np.linalg.norm(ref) == 0:
            assert np.all(out[b] == 0)
        else:
            assert rel(out[b], ref) < SVST_TOL[form], (b, rel(out[b], ref))


@pytest.mark.parametrize("form", ["plain", "tuned"])
def test_svst_batch_full_scale(torch, M, form):
    """The 10³ scale of the workload as one batch: 486 patches of 1000 × 300
    (Gram side 300), rank-8 signal + noise, thresholds inside the spectrum;
    three patches (first, middle, last) against the FP64 oracle."""
    m, n, batch = 1000, 300, 486
    rng = np.random.default_rng(486)
    X = (rng.standard_normal((batch, m, n)) + 1j * rng.standard_normal((batch, m, n))).astype(np.complex64)
    U = rng.standard_normal((batch, m, 8)) + 1j * rng.standard_normal((batch, m, 8))
    V = rng.standard_normal((batch, 8, n)) + 1j * rng.standard_normal((batch, 8, n))
    X += (4.0 * np.einsum("bij,bjk->bik", U, V)).astype(np.complex64)
    betas = [40.0 + (b % 7) for b in range(batch)]
    cm = np.ascontiguousarray(np.transpose(X, (0, 2, 1)))
    from mslr_recon_b200.context import FORMS
    out = M.svst_batch(dev(torch, cm), m, n, betas, form=FORMS[form]).cpu().numpy()
    out = np.transpose(out, (0, 2, 1))
    for b in (0, batch // 2, batch - 1):
        ref = O.svst(X[b].astype(np.complex128), betas[b])
        assert rel(out[b], ref) < SVST_TOL[form], (b, rel(out[b], ref))


@pytest.mark.parametrize("form", ["plain", "tuned"])
def test_svst_batch_full_rank(torch, M, form):
    """Every singular value above the threshold, as in the metric workload's
    POGM iterates: 48 patches of 1000 × 300 (Gram side 300) with a small β,
    so that all 300 eigenvectors of every patch are back-transformed; three
    patches against the FP64 oracle."""
    m, n, batch = 1000, 300, 48
    rng = np.random.default_rng(300)
    X = (rng.standard_normal((batch, m, n)) + 1j * rng.standard_normal((batch, m, n))).astype(np.complex64)
    betas = [2.0 + 0.1 * (b % 5) for b in range(batch)]
    assert min(np.linalg.svd(X[0], compute_uv=False)) > max(betas)
    cm = np.ascontiguousarray(np.transpose(X, (0, 2, 1)))
    from mslr_recon_b200.context import FORMS
    out = M.svst_batch(dev(torch, cm), m, n, betas, form=FORMS[form]).cpu().numpy()
    out = np.transpose(out, (0, 2, 1))
    for b in (0, batch // 2, batch - 1):
        ref = O.svst(X[b].astype(np.complex128), betas[b])
        assert rel(out[b], ref) < SVST_TOL[form], (b, rel(out[b], ref))


def test_svst_single_matrix(torch, M):
    rng = np.random.default_rng(12)
    X = (rng.standard_normal((50, 20)) + 1j * rng.standard_normal((50, 20))).astype(np.complex64)
    out = M.SVST(dev(torch, X), 4.0).cpu().numpy()
    assert rel(out, O.svst(X.astype(np.complex128), 4.0)) < SVST_TOL["tuned"]   # default form


@pytest.mark.parametrize("k", [0, 1, 2])
def test_patch_svst_golden(torch, M, gold, k):
    out = M.patchSVST(dev(torch, gold["x"]), 3.0, PATCHES[k], STRIDES[k]).cpu().numpy()
    assert rel(out, gold[f"svst{k}"]) < SVST_TOL["tuned"]   # default form


# --- SENSE -------------------------------------------------------------------------
@pytest.fixture(scope="module")
def gctx(torch, M, gold):
    Nt, Nc, K = gold["y"].shape
    ctx = M.MSLRContext((8, 6, 4), Nc, Nt, K, PATCHES, STRIDES, form="plain")
    ctx.bind(dev(torch, gold["smaps"]), dev(torch, gold["y"]), dev(torch, gold["idx"], torch.int32))
    yield ctx
    ctx.close()


def test_sense_forward_golden(torch, gctx, gold):
    y = gctx.forward(dev(torch, gold["x"])).cpu().numpy()
    assert rel(y, gold["Ax"]) < 1e-5


def test_sense_adjoint_golden(torch, gctx, gold):
    x = gctx.adjoint(dev(torch, gold["y"])).cpu().numpy()
    assert rel(x, gold["AHy"]) < 1e-5


def test_normal_op_matches_forward_adjoint(torch, gctx, gold):
    X = np.stack([gold["x"], 0.5 * gold["x"]]).astype(np.complex64)
    g = gctx.normal(dev(torch, X)).cpu().numpy()
    xs = X.astype(np.complex128).sum(0)
    smaps, idx = gold["smaps"], gold["idx"]
    ref = O.sense_adjoint(O.sense_forward(xs, smaps, idx) - gold["y"], smaps, idx)
    assert rel(g, ref) < 1e-5


def test_patch_svst_context_golden(torch, gctx, gold):
    for k in range(3):
        out = gctx.patch_svst(k, 3.0, dev(torch, gold["x"])).cpu().numpy()
        assert rel(out, gold[f"svst{k}"]) < 2e-5, k


# --- POGM ---------------------------------------------------------------------------
def test_pogm_trajectory_golden(torch, gctx, gold):
    X = gctx.init_x0()
    traj = gold["traj"]
    niter = traj.shape[0]
    gctx.pogm_begin(X, niter, L=3.0)
    errs = []
    for i in range(niter):
        gctx.pogm_step(X)
        errs.append(rel(X.cpu().numpy(), traj[i]))
    assert max(errs) < 1e-4, errs
    assert gctx.pogm_restarts() == [bool(v) for v in gold["restarts"]]


def test_power_iteration(torch, gctx, gold):
    s1, it = gctx.power_iter(200, 1e-6)
    smaps, idx = gold["smaps"], gold["idx"]
    _, ref = O.poweriter_mod(lambda v: O.sense_forward(v, smaps, idx),
                             lambda v: O.sense_adjoint(v, smaps, idx),
                             np.ones(gold["x"].shape, complex), niter=200, tol=1e-6)
    assert s1 == pytest.approx(ref, rel=1e-4)


def test_small_workload_per_iteration_parity(torch, M, small_problem):
    """The small workload (32x32x24, 8 coils, Nt=64, one 6^3 scale with
    clamped edge patches, 20 iterations): X after every iteration within 1e-4
    of the FP64 oracle, identical restart flags."""
    pb = small_problem
    Nt, Nc, K = pb["y"].shape
    niter = pb["niters"]
    prob = O.ReconProblem(smaps=pb["smaps"].astype(np.complex128), idx=pb["idx"],
                          y=pb["y"].astype(np.complex128), patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"], sigma1=1.0)
    traj = []
    _, restarts, _, _ = O.run_recon_arrays(prob, niter, iter_callback=lambda it, xk, r: traj.append(xk.copy()))
    for form in ("plain", "tuned"):
        with M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form=form) as ctx:
            ctx.bind(dev(torch, pb["smaps"]), dev(torch, pb["y"]), dev(torch, pb["idx"], torch.int32))
            X = ctx.init_x0()
            ctx.pogm_begin(X, niter, L=1.0)
            errs = []
            for i in range(niter):
                ctx.pogm_step(X)
                errs.append(rel(X.cpu().numpy(), traj[i]))
            assert max(errs) < 1e-4, (form, errs)
            assert ctx.pogm_restarts() == restarts, form


@pytest.mark.parametrize("form", ["plain", "tuned"])
def test_costs_per_iteration_vs_oracle(torch, M, small_problem, form):
    """run_recon's logged costs (dc_cost, reg_cost at X0 and after every
    iteration, scripts/reconstruct.jl:176-205) against the FP64 oracle on the
    small workload, within 1e-4 relative."""
    pb = small_problem
    niter = 6
    prob = O.ReconProblem(smaps=pb["smaps"].astype(np.complex128), idx=pb["idx"],
                          y=pb["y"].astype(np.complex128), patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"], sigma1=1.0)
    _, _, dcs, regs = O.run_recon_arrays(prob, niter, log_costs=True)
    out = M.run_recon(pb["smaps"], pb["y"], pb["idx"], pb["patch_sizes"], pb["strides"], niter,
                      sigma1=1.0, form=form, log_costs=True, return_components=False)
    assert len(out["dc_costs"]) == niter + 1 == len(dcs)
    for a, b in zip(out["dc_costs"], dcs):
        assert a == pytest.approx(b, rel=1e-4), (form, out["dc_costs"], dcs)
    for a, b in zip(out["reg_costs"], regs):
        assert a == pytest.approx(b, rel=1e-4), (form, out["reg_costs"], regs)


def test_graph_replay_is_bit_identical(torch, M, small_problem):
    """Tuned form: the graph-captured iteration (default) and direct kernel
    launches give bit-identical iterates and restart flags, and the graph is
    re-captured when the iterate moves to another buffer."""
    pb = small_problem
    Nt, Nc, K = pb["y"].shape
    outs = []
    for graph in (True, False):
        with M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form="tuned") as ctx:
            ctx.set_graph(graph)
            ctx.bind(dev(torch, pb["smaps"]), dev(torch, pb["y"]), dev(torch, pb["idx"], torch.int32))
            X = ctx.init_x0()
            ctx.pogm_begin(X, 6, L=1.0)
            for _ in range(3):
                ctx.pogm_step(X)
            X2 = X.clone()              # continue on another buffer
            for _ in range(3):
                ctx.pogm_step(X2)
            torch.cuda.synchronize()
            outs.append((X2.cpu().numpy(), ctx.pogm_restarts()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1]


# --- errors -------------------------------------------------------------------------
def test_bad_indices_rejected(torch, M, gold):
    Nt, Nc, K = gold["y"].shape
    with M.MSLRContext((8, 6, 4), Nc, Nt, K, PATCHES[:1], STRIDES[:1]) as ctx:
        idx = gold["idx"].copy()
        idx[0, 3] = idx[0, 2]   # duplicate -> not strictly ascending
        with pytest.raises(ValueError, match="ascending"):
            ctx.bind(dev(torch, gold["smaps"]), dev(torch, gold["y"]), dev(torch, idx, torch.int32))
        idx = gold["idx"].copy()
        idx[1, -1] = 8 * 6 * 4
        with pytest.raises(ValueError, match="range"):
            ctx.bind(dev(torch, gold["smaps"]), dev(torch, gold["y"]), dev(torch, idx, torch.int32))


def test_state_errors(torch, M, gold):
    Nt, Nc, K = gold["y"].shape
    with M.MSLRContext((8, 6, 4), Nc, Nt, K, PATCHES[:1], STRIDES[:1]) as ctx:
        with pytest.raises(M.MSLRError, match="bind"):
            ctx.forward(dev(torch, gold["x"]))


@pytest.mark.parametrize("form", ["plain", "tuned"])
@pytest.mark.parametrize("N,Nc", [((90, 90, 60), 18), ((48, 48, 32), 12), ((45, 30, 20), 5),
                                  ((32, 32, 24), 8), ((8, 6, 4), 3)])
def test_sense_metric_shapes(torch, M, form, N, Nc):
    """Forward, adjoint and normal operator at the benchmark image shapes
    (two-pass radix plans in the tuned kernels; an odd axis included)."""
    ctx_form = "tuned" if form.startswith("tuned") else form
    rng = np.random.default_rng(sum(N) + Nc)
    Nx, Ny, Nz = N
    Nt = 3
    nvox = Nx * Ny * Nz
    K = nvox // 6
    smaps = (rng.standard_normal((Nc, Nz, Ny, Nx)) + 1j * rng.standard_normal((Nc, Nz, Ny, Nx)))
    smaps /= np.sqrt(np.sum(np.abs(smaps) ** 2, axis=0))[None]
    idx = np.stack([np.sort(rng.choice(nvox, K, replace=False)) for _ in range(Nt)]).astype(np.int32)
    x = rng.standard_normal((Nt, Nz, Ny, Nx)) + 1j * rng.standard_normal((Nt, Nz, Ny, Nx))
    y = rng.standard_normal((Nt, Nc, K)) + 1j * rng.standard_normal((Nt, Nc, K))
    with M.MSLRContext(N, Nc, Nt, K, [[Nx, Ny, Nz]], [[Nx, Ny, Nz]], form=ctx_form) as ctx:
        ctx.bind(dev(torch, smaps), dev(torch, y), dev(torch, idx, torch.int32))
        yf = ctx.forward(dev(torch, x)).cpu().numpy()
        assert rel(yf, O.sense_forward(x, smaps, idx)) < 1e-5
        xa = ctx.adjoint(dev(torch, y)).cpu().numpy()
        assert rel(xa, O.sense_adjoint(y, smaps, idx)) < 1e-5
        g = ctx.normal(dev(torch, x[None])).cpu().numpy()
        ref = O.sense_adjoint(O.sense_forward(x, smaps, idx) - y, smaps, idx)
        assert rel(g, ref) < NORMAL_TOL[form], rel(g, ref)


def test_normal_op_tensor_core_plane_pass(torch, M, monkeypatch):
    """The optional plane pass of the tuned normal operator as tcgen05 DFT
    products (MSLR_XY_PATH=tc) at 90×90×60: within 5e-5 of the FP64 oracle
    (split-BF16 products), and the POGM-facing forward / adjoint unchanged."""
    monkeypatch.setenv("MSLR_XY_PATH", "tc")
    test_sense_metric_shapes(torch, M, "tuned-tc", (90, 90, 60), 18)


@pytest.mark.parametrize("path", ["four", "four-one-lane", "three"])
@pytest.mark.parametrize("aligned", [True, False])
def test_normal_op_summed_scales(torch, M, monkeypatch, path, aligned):
    """g = A'(A Σ_k X_k − y) for two scale images at 90×90×60, 18 coils and
    two chunks of frames: the four-pass form (summed image by k_xsum, then
    the four chunk kernels, chunks on two streams or, with
    MSLR_SENSE_LANES=1, on one) and the three-kernel form
    (MSLR_SENSE_PATH=3), with X 16-byte aligned or not, against the FP64
    oracle."""
    if path == "three":
        monkeypatch.setenv("MSLR_SENSE_PATH", "3")
    if path == "four-one-lane":
        monkeypatch.setenv("MSLR_SENSE_LANES", "1")
    rng = np.random.default_rng(77)
    N, Nc, Nt = (90, 90, 60), 18, 5
    Nx, Ny, Nz = N
    nvox = Nx * Ny * Nz
    K = nvox // 6
    smaps = rng.standard_normal((Nc, Nz, Ny, Nx)) + 1j * rng.standard_normal((Nc, Nz, Ny, Nx))
    smaps /= np.sqrt(np.sum(np.abs(smaps) ** 2, axis=0))[None]
    idx = np.stack([np.sort(rng.choice(nvox, K, replace=False)) for _ in range(Nt)]).astype(np.int32)
    X = rng.standard_normal((2, Nt, Nz, Ny, Nx)) + 1j * rng.standard_normal((2, Nt, Nz, Ny, Nx))
    y = rng.standard_normal((Nt, Nc, K)) + 1j * rng.standard_normal((Nt, Nc, K))
    with M.MSLRContext(N, Nc, Nt, K, [[Nx, Ny, Nz], [10, 10, 10]], [[Nx, Ny, Nz], [10, 10, 10]],
                       form="tuned") as ctx:
        ctx.bind(dev(torch, smaps), dev(torch, y), dev(torch, idx, torch.int32))
        Xd = dev(torch, X)
        if not aligned:   # the same values 8 bytes past a 16-byte boundary
            flat = torch.empty(1 + Xd.numel(), dtype=torch.complex64, device=Xd.device)
            Xd = flat[1:].view(Xd.shape).copy_(Xd)
            assert Xd.data_ptr() % 16 == 8
        g = ctx.normal(Xd).cpu().numpy()
        xs = X.sum(axis=0)
        ref = O.sense_adjoint(O.sense_forward(xs, smaps, idx) - y, smaps, idx)
        assert rel(g, ref) < 1e-5, rel(g, ref)
        kms, _ = ctx.normal_profile(Xd)
        assert set(kms) == ({"pfwd", "zmask", "padj", "csum"} if path.startswith("four")
                            else {"zfwd", "xy", "zadj"})


@pytest.mark.parametrize("form", ["plain", "tuned"])
def test_per_patch_thresholds_and_nucnorm(torch, M, form):
    """patchSVST with one λ per patch and both patch_nucnorm forms
    (src/recon.jl:138-166, :263-268) on a grid with overlapping and clamped
    patches, against the FP64 oracle."""
    rng = np.random.default_rng(31)
    N, Nt = (13, 11, 9), 20
    ps, ss = [4, 4, 4], [3, 3, 3]
    Nx, Ny, Nz = N
    img = (rng.standard_normal((Nt, Nz, Ny, Nx)) + 1j * rng.standard_normal((Nt, Nz, Ny, Nx))).astype(np.complex64)
    g = O.patch_geometry(N, ps, ss)
    lams = rng.uniform(0.5, 6.0, g.Np)
    with M.MSLRContext(N, 2, Nt, 10, [ps], [ss], form=form) as ctx:
        out = ctx.patch_svst_lambdas(0, lams, dev(torch, img)).cpu().numpy()
        ref = O.patch_svst(img.astype(np.complex128), lams, ps, ss)
        assert rel(out, ref) < SVST_TOL[form], rel(out, ref)
        P = O.img2patches(img.astype(np.complex128), ps, ss)
        assert ctx.patch_nucnorm(0, dev(torch, img)) == pytest.approx(O.patch_nucnorm(P), rel=1e-5)
        assert ctx.patch_nucnorm(0, dev(torch, img), lams) == pytest.approx(
            O.patch_nucnorm_weighted(P, lams), rel=1e-5)


def test_contexts_of_different_shapes_coexist(torch, M, gold):
    """A context created after another one of a smaller image shape leaves
    the first one's kernels launchable: the kernels' shared-memory limits are
    per process and only ever raised."""
    Nt, Nc, K = gold["y"].shape
    rng = np.random.default_rng(3)
    N = (32, 32, 24)
    nvox = 32 * 32 * 24
    smaps = rng.standard_normal((Nc, 24, 32, 32)) + 1j * rng.standard_normal((Nc, 24, 32, 32))
    idx = np.stack([np.sort(rng.choice(nvox, 500, replace=False)) for _ in range(2)]).astype(np.int32)
    y = rng.standard_normal((2, Nc, 500)) + 1j * rng.standard_normal((2, Nc, 500))
    with M.MSLRContext(N, Nc, 2, 500, [[8, 8, 8]], [[8, 8, 8]]) as big, \
            M.MSLRContext((32, 32, 8), 1, 2, 1, [[8, 8, 8]], [[8, 8, 8]]) as small:
        big.bind(dev(torch, smaps), dev(torch, y), dev(torch, idx, torch.int32))
        xa = big.adjoint(dev(torch, y)).cpu().numpy()
        assert rel(xa, O.sense_adjoint(y, smaps, idx)) < 1e-5
        assert small.N == (32, 32, 8)


def test_mixed_gram_sides_per_iteration(torch, M):
    """Scales whose Gram sides need both eigen variants (400 > 384 and 64) in
    one tuned-form iteration: X after every iteration within 1e-4 of the FP64
    oracle, identical restart flags."""
    rng = np.random.default_rng(31)
    N, Nc, Nt = (16, 16, 8), 2, 400
    nvox = N[0] * N[1] * N[2]
    K = nvox // 3
    smaps = rng.standard_normal((Nc, N[2], N[1], N[0])) + 1j * rng.standard_normal((Nc, N[2], N[1], N[0]))
    smaps /= np.sqrt((np.abs(smaps) ** 2).sum(0))[None]
    idx = np.stack([np.sort(rng.choice(nvox, K, replace=False)) for _ in range(Nt)]).astype(np.int32)
    U = rng.standard_normal((nvox, 3)) + 1j * rng.standard_normal((nvox, 3))
    V = rng.standard_normal((Nt, 3)) + 1j * rng.standard_normal((Nt, 3))
    x = (V @ U.T).reshape(Nt, N[2], N[1], N[0]) * 10
    y = O.sense_forward(x, smaps, idx) + 0.05 * (rng.standard_normal((Nt, Nc, K)) + 1j * rng.standard_normal((Nt, Nc, K)))
    ps = [[16, 16, 8], [4, 4, 4]]
    prob = O.ReconProblem(smaps=smaps, idx=idx, y=y, patch_sizes=ps, strides=ps, sigma1=1.0)
    traj = []
    _, restarts, _, _ = O.run_recon_arrays(prob, 3, iter_callback=lambda it, xk, r: traj.append(xk.copy()))
    with M.MSLRContext(N, Nc, Nt, K, ps, ps, form="tuned") as ctx:
        ctx.bind(dev(torch, smaps), dev(torch, y), dev(torch, idx, torch.int32))
        X = ctx.init_x0()
        ctx.pogm_begin(X, 3, L=2.0)
        errs = []
        for i in range(3):
            ctx.pogm_step(X)
            errs.append(rel(X.cpu().numpy(), traj[i]))
        assert max(errs) < 1e-4, errs
        assert ctx.pogm_restarts() == restarts


def test_autotune_keeps_parity(torch, M, small_problem):
    """The autotuner's choices (SENSE chunk shape, lanes and z-mask variant,
    Gram split counts, eigen CTA variants) are valid and the tuned iteration
    still matches the FP64 oracle."""
    pb = small_problem
    Nt, Nc, K = pb["y"].shape
    niter = 6
    prob = O.ReconProblem(smaps=pb["smaps"].astype(np.complex128), idx=pb["idx"],
                          y=pb["y"].astype(np.complex128), patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"], sigma1=1.0)
    traj = []
    _, restarts, _, _ = O.run_recon_arrays(prob, niter, iter_callback=lambda it, xk, r: traj.append(xk.copy()))
    with M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form="tuned") as ctx:
        ctx.bind(dev(torch, pb["smaps"]), dev(torch, pb["y"]), dev(torch, pb["idx"], torch.int32))
        t = ctx.autotune()
        assert t["coils_per_group"] in (2, 3, 4, 6, 8) and 1 <= t["frames_per_chunk"] <= 4
        assert len(t["gram_splits"]) == len(pb["patch_sizes"])
        assert t["lanes"] in (1, 2) and t["zmask_ctas_per_sm"] in (1, 2)
        assert len(t["eig_threads"]) == len(pb["patch_sizes"])
        assert all(v in (384, 1024) for v in t["eig_threads"])
        X = ctx.init_x0()
        ctx.pogm_begin(X, niter, L=1.0)
        errs = []
        for i in range(niter):
            ctx.pogm_step(X)
            errs.append(rel(X.cpu().numpy(), traj[i]))
        assert max(errs) < 1e-4, errs
        assert ctx.pogm_restarts() == restarts


@pytest.mark.parametrize("form", ["plain", "tuned"])
@pytest.mark.parametrize("N,Nt,bsig", [((9, 9, 9), 5, 0.7), ((12, 10, 8), 6, 0.5)])
def test_pogm_bsig_and_odd_sizes(torch, M, form, N, Nt, bsig):
    """POGM with σ decay (bsig < 1: the gradient-sign test and its previous-
    gradient buffer) on an image × frames count that is odd (element-wise
    update path) and even (paired update path): every iterate within 1e-4 of
    the FP64 oracle, identical restart flags."""
    rng = np.random.default_rng(sum(N) + Nt)
    Nc = 3
    nvox = N[0] * N[1] * N[2]
    K = nvox // 2
    smaps = rng.standard_normal((Nc, N[2], N[1], N[0])) + 1j * rng.standard_normal((Nc, N[2], N[1], N[0]))
    smaps /= np.sqrt((np.abs(smaps) ** 2).sum(0))[None]
    idx = np.stack([np.sort(rng.choice(nvox, K, replace=False)) for _ in range(Nt)]).astype(np.int32)
    x = (rng.standard_normal((Nt, nvox, 2)) @ rng.standard_normal((2, 1)))[..., 0].reshape(Nt, N[2], N[1], N[0])
    y = O.sense_forward(x + 0j, smaps, idx) + 0.1 * (rng.standard_normal((Nt, Nc, K)) + 1j * rng.standard_normal((Nt, Nc, K)))
    ps = [list(N), [3, 3, 2]]
    prob = O.ReconProblem(smaps=smaps, idx=idx, y=y, patch_sizes=ps, strides=ps, sigma1=1.0)
    niter = 8
    traj = []
    _, restarts, _, _ = O.run_recon_arrays(prob, niter, bsig=bsig,
                                           iter_callback=lambda it, xk, r: traj.append(xk.copy()))
    with M.MSLRContext(N, Nc, Nt, K, ps, ps, form=form) as ctx:
        ctx.bind(dev(torch, smaps), dev(torch, y), dev(torch, idx, torch.int32))
        X = ctx.init_x0()
        ctx.pogm_begin(X, niter, L=2.0, bsig=bsig)
        errs = []
        for i in range(niter):
            ctx.pogm_step(X)
            errs.append(rel(X.cpu().numpy(), traj[i]))
        assert max(errs) < 1e-4, errs
        assert ctx.pogm_restarts() == restarts
