"""The oracle's restatement of run_recon's data set-up
(scripts/reconstruct.jl:86-147): maps normalisation, the 99th-percentile
sense_comb scaling, the mask taken from coil 1 with its two checks, the
gathered samples — against the synthetic generator, which builds its problems
with the same conventions."""
import importlib.util
import os
import sys

import numpy as np
import pytest

from oracle import mslr_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def synth():
    spec = importlib.util.spec_from_file_location("mslr_synth_setup",
                                                  os.path.join(os.path.dirname(HERE), "mslr-recon_b200",
                                                               "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def raw_inputs(seed=0):
    S = synth()
    cfg = S.SynthConfig(N=(12, 10, 8), Nc=4, Nt=5, rank=2, frac=0.3, centre=4, seed=300 + seed,
                        normalize=False)
    pb = S.make_problem(cfg)
    Nt, Nc, K = pb["y"].shape
    Nx, Ny, Nz = pb["N"]
    ksp = np.zeros((Nt, Nc, Nz * Ny * Nx), np.complex64)
    for t in range(Nt):
        ksp[t][:, pb["idx"][t]] = pb["y"][t]
    rng = np.random.default_rng(seed)
    w = (0.5 + rng.random((Nz, Ny, Nx))).astype(np.float32)   # un-normalise the maps
    smaps_raw = (pb["smaps"] * w[None]).astype(np.complex64)
    return S, pb, ksp.reshape(Nt, Nc, Nz, Ny, Nx), smaps_raw


def test_prepare_matches_generator():
    S, pb, ksp, smaps_raw = raw_inputs()
    smaps, y, idx, scale = O.prepare_kspace(ksp, smaps_raw)
    assert np.array_equal(idx, pb["idx"])
    assert O.rel_err(smaps, pb["smaps"]) < 1e-6
    ref_scale = S.sense_comb_scale(pb["y"], pb["smaps"], pb["idx"])
    assert scale == pytest.approx(ref_scale, rel=1e-5)
    assert O.rel_err(y, pb["y"] / np.float32(scale)) < 1e-6


def test_quantile_type7():
    v = np.array([3.0, 1.0, 4.0, 1.0, 5.0, 9.0, 2.0, 6.0], np.float32)
    for p in (0.0, 0.25, 0.5, 0.99, 1.0):
        assert O.quantile_type7(v, p) == pytest.approx(float(np.quantile(v.astype(np.float64), p)), rel=1e-7)


def test_prepare_rejects_coil_with_other_pattern():
    _, _, ksp, smaps_raw = raw_inputs(1)
    bad = ksp.copy()
    nz = np.flatnonzero(bad[2, 2].ravel())
    bad[2, 2].reshape(-1)[nz[0]] = 0
    with pytest.raises(O.SetupError, match="Coil 3 has a different sampling pattern"):
        O.prepare_kspace(bad, smaps_raw)


def test_prepare_rejects_frame_with_other_count():
    _, _, ksp, smaps_raw = raw_inputs(2)
    bad = ksp.copy()
    nz = np.flatnonzero(bad[3, 0].ravel())
    bad[3, :].reshape(bad.shape[1], -1)[:, nz[0]] = 0
    with pytest.raises(O.SetupError, match="Frame 4 has a different sample count"):
        O.prepare_kspace(bad, smaps_raw)
