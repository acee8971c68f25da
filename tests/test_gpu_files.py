"""run_recon with its files (scripts/reconstruct.jl:58-263): the coil maps
read with matread, the zero-filled k-space ``ksp_epi_zf`` with h5read, the
reconstruction on the device, and the results written with matwrite — the
sixteen variables the reference saves, checked against the in-memory
reconstruction on the same arrays (bit-exact) and X against the FP64
oracle's reconstruction from the oracle's own set-up (1e-4 relative)."""
import numpy as np
import pytest

from oracle import mslr_oracle as O
from tests.test_setup_oracle import raw_inputs

pytestmark = pytest.mark.gpu

SAVED = {"X", "X_recon", "omega", "dc_costs", "reg_costs", "restarts", "R", "sigma1A", "L", "Nscales",
         "patch_sizes", "strides", "lambdas", "Niters", "scale_factor", "used_gpu"}


@pytest.mark.parametrize("compress", [False, True])
def test_run_recon_files_end_to_end(tmp_path, compress):
    import torch
    assert torch.cuda.is_available()
    import mslr_recon_b200 as M
    from mslr_recon_b200.matio import h5read, matread, matwrite

    _, pb, ksp, smaps_raw = raw_inputs(5)
    Nt, Nc, Nz, Ny, Nx = ksp.shape
    ps = [list(pb["N"]), [4, 5, 4]]
    niters = 4
    fn_smaps, fn_ksp = str(tmp_path / "smaps.mat"), str(tmp_path / "ksp.mat")
    matwrite(fn_smaps, {"smaps": smaps_raw}, compress=compress)
    matwrite(fn_ksp, {"ksp_epi_zf": ksp}, compress=compress, chunk_bytes=1 << 14)
    assert np.array_equal(h5read(fn_ksp, "ksp_epi_zf"), ksp)

    fn_out, out = M.run_recon_files(fn_ksp, fn_smaps, str(tmp_path / "recon"), N=pb["N"], Nvc=Nc, Nt=Nt,
                                    PATCH_SIZES=ps, STRIDES=ps, NITERS=niters, sigma1A_precomputed=1.0,
                                    form="tuned", compress=compress)
    assert fn_out.endswith("recon_2scales.mat")
    ref = M.run_recon_kspace(ksp, smaps_raw, ps, ps, niters, sigma1=1.0, form="tuned", log_costs=True)
    r = matread(fn_out)
    assert set(r) == SAVED
    assert r["X"].shape == (2, Nt, Nz, Ny, Nx) and r["X"].dtype == np.complex64
    assert np.array_equal(r["X"], ref["X"])
    assert np.array_equal(r["X_recon"], ref["X_recon"])
    assert np.array_equal(r["dc_costs"].ravel(), np.asarray(ref["dc_costs"]))
    assert np.array_equal(r["reg_costs"].ravel(), np.asarray(ref["reg_costs"]))
    assert r["restarts"].ravel().tolist() == list(ref["restarts"])
    omega = ksp[:, 0] != 0
    assert np.array_equal(r["omega"], omega)
    assert r["R"] == pytest.approx(Nx * Ny * Nz / omega[0].sum(), rel=1e-15)
    assert r["Nscales"] == 2 and r["Niters"] == niters and r["used_gpu"] is True
    assert [p.ravel().tolist() for p in r["patch_sizes"]] == ps
    assert r["lambdas"].ravel().tolist() == pytest.approx(ref["lambdas"], rel=1e-15)
    assert r["scale_factor"] == pytest.approx(ref["scale_factor"], rel=1e-6)

    # the oracle's own set-up and FP64 reconstruction
    smaps, y, idx, _ = O.prepare_kspace(ksp, smaps_raw)
    prob = O.ReconProblem(smaps=smaps, idx=idx, y=y, patch_sizes=ps, strides=ps, sigma1=1.0)
    X_o, restarts_o, _, _ = O.run_recon_arrays(prob, niters)
    assert O.rel_err(r["X"], X_o) < 1e-4
