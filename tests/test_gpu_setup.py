"""run_recon's data set-up on the device (mslr_sos_normalize, mslr_sampling,
mslr_prepare) against the oracle's restatement of
scripts/reconstruct.jl:86-147: normalised maps and sample indices bit-exact,
scale factor and scaled samples to FP32 rounding, the reference's assertion
messages, and a whole reconstruction from raw inputs equal to one from the
prepared inputs."""
import numpy as np
import pytest

from oracle import mslr_oracle as O
from tests.test_setup_oracle import raw_inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def M():
    import mslr_recon_b200 as M
    return M


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("seed", [0, 3])
def test_prepare_matches_oracle(torch, M, seed):
    _, pb, ksp, smaps_raw = raw_inputs(seed)
    sm_o, y_o, idx_o, sf_o = O.prepare_kspace(ksp, smaps_raw)
    Nt, Nc = ksp.shape[:2]
    K = M.sampling(dev(torch, ksp))
    assert K == idx_o.shape[1]
    with M.MSLRContext(pb["N"], Nc, Nt, K, [list(pb["N"])], [list(pb["N"])]) as ctx:
        smaps, y, idx, sf = ctx.prepare(dev(torch, ksp), dev(torch, smaps_raw))
    assert np.array_equal(smaps.cpu().numpy(), sm_o)
    assert np.array_equal(idx.cpu().numpy(), idx_o)
    assert sf == pytest.approx(sf_o, rel=1e-5)
    assert O.rel_err(y.cpu().numpy(), y_o) < 1e-6


def test_sos_normalize_bit_exact(torch, M):
    _, pb, _, smaps_raw = raw_inputs(4)
    Nc, Nz, Ny, Nx = smaps_raw.shape
    from mslr_recon_b200._lib import check, i32arr, lib
    src = dev(torch, smaps_raw)
    out = torch.empty_like(src)
    check(lib.mslr_sos_normalize(i32arr([Nx, Ny, Nz]), Nc, src.data_ptr(), out.data_ptr(), None))
    assert np.array_equal(out.cpu().numpy(), O.sos_normalize_maps(smaps_raw))


def test_sampling_rejects_bad_patterns(torch, M):
    _, _, ksp, _ = raw_inputs(1)
    bad = ksp.copy()
    nz = np.flatnonzero(bad[2, 2].ravel())
    bad[2, 2].reshape(-1)[nz[0]] = 0
    with pytest.raises(ValueError, match="Coil 3 has a different sampling pattern"):
        M.sampling(dev(torch, bad))
    bad = ksp.copy()
    nz = np.flatnonzero(bad[3, 0].ravel())
    bad[3, :].reshape(bad.shape[1], -1)[:, nz[0]] = 0
    with pytest.raises(ValueError, match="Frame 4 has a different sample count"):
        M.sampling(dev(torch, bad))


def test_run_recon_from_raw_inputs(torch, M):
    _, pb, ksp, smaps_raw = raw_inputs(5)
    ps = [list(pb["N"]), [4, 5, 4]]
    raw = M.run_recon_kspace(ksp, smaps_raw, ps, ps, niters=4, sigma1=1.0, form="plain")
    ref = M.run_recon(raw["smaps"], raw["y"], raw["idx"], ps, ps, niters=4, sigma1=1.0, form="plain")
    assert np.array_equal(raw["X"], ref["X"])
    assert raw["restarts"] == ref["restarts"]
