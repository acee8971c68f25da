"""Generate tests/golden/golden_small.npz from the CPU oracle.

The reference (Julia) ships no golden vectors and cannot run here, so these
fixtures are produced by the oracle itself on tiny seeded inputs; they pin
the oracle against regressions and give the GPU tests fixed expected
outputs.  Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import mslr_oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_small.npz")

N = (8, 6, 4)          # (Nx, Ny, Nz) — odd-free but non-power-of-two
NC, NT, K = 3, 10, 90
PATCHES = [[8, 6, 4], [4, 3, 2], [3, 3, 3]]
STRIDES = [[8, 6, 4], [4, 3, 2], [2, 2, 2]]   # global, partition, overlapping + clamped
NITER = 6


def problem():
    rng = np.random.Generator(np.random.PCG64(20251106))
    Nx, Ny, Nz = N
    nvox = Nx * Ny * Nz

    def cn(*s):
        return (rng.standard_normal(s) + 1j * rng.standard_normal(s)) / np.sqrt(2)

    smaps = cn(NC, Nz, Ny, Nx)
    smaps /= np.sqrt(np.sum(np.abs(smaps) ** 2, axis=0))[None]
    idx = np.stack([np.sort(rng.choice(nvox, K, replace=False)) for _ in range(NT)]).astype(np.int32)
    M = cn(nvox, 2) * 8.0
    B, _ = np.linalg.qr(cn(NT, 2))
    x = (np.conj(B) @ M.T).reshape(NT, Nz, Ny, Nx) + 0.3 * cn(NT, Nz, Ny, Nx)
    y = O.sense_forward(x, smaps, idx) + 0.05 * cn(NT, NC, K)
    return smaps, idx, y, x


def compute():
    smaps, idx, y, x = problem()
    out = {"smaps": smaps, "idx": idx, "y": y, "x": x}
    out["Ax"] = O.sense_forward(x, smaps, idx)
    out["AHy"] = O.sense_adjoint(y, smaps, idx)
    # patch geometry and extract/recombine for each scale
    for k, (ps, ss) in enumerate(zip(PATCHES, STRIDES)):
        g = O.patch_geometry(N, ps, ss)
        out[f"starts{k}"] = np.concatenate([np.array(s) for s in g.starts]).astype(np.int32)
        P = O.img2patches(x, ps, ss)
        out[f"P{k}"] = P
        out[f"recomb{k}"] = O.patches2img(P, ps, ss, N)
        out[f"svst{k}"] = O.patch_svst(x, 3.0, ps, ss)
    prob = O.ReconProblem(smaps=smaps, idx=idx, y=y, patch_sizes=PATCHES, strides=STRIDES,
                          sigma1=1.0, workers=1)
    traj = []
    Xf, restarts, _, _ = O.run_recon_arrays(prob, NITER, iter_callback=lambda it, xk, r: traj.append(xk.copy()))
    out["traj"] = np.stack(traj)
    out["restarts"] = np.array(restarts, dtype=np.uint8)
    return out


if __name__ == "__main__":
    np.savez_compressed(OUT, **compute())
    print("wrote", OUT)
