"""Generate tests/golden/grad_diff.npz: the FP64 oracle's loss and gradient
d loss / d log λ_k of the unrolled POGM at the differentiation workload
(48×48×32, 12 coils, Nt = 128, scales [48,48,32] and [8,8,8] with equal
strides, 10 iterations, L = 2, the synthetic generator's "diff" problem built
with scipy FFTs), together with FP64 central finite differences of the
oracle's forward at h = 1e-3 in log λ_k.  The oracle's reverse accumulation
is itself checked against finite differences on small problems in
tests/test_grad_oracle.py.  Run:  python tests/golden/make_grad_golden.py
(about ten minutes on eight cores)."""
import importlib.util
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import mslr_oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "grad_diff.npz")
NITER = 10
L = 2.0
H = 1e-3


def synth():
    spec = importlib.util.spec_from_file_location("mslr_synth_golden",
                                                  os.path.join(ROOT, "mslr-recon_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    S = synth()
    pb = S.make_problem(S.CONFIGS["diff"])
    prob = O.ReconProblem(smaps=pb["smaps"].astype(np.complex128), idx=pb["idx"],
                          y=pb["y"].astype(np.complex128), patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"])
    Xt = pb["x_true"].astype(np.complex128)
    lam = np.array(prob.lambdas())
    loss, grad, _, restarts = O.pogm_unrolled_grad(prob, NITER, Xt, list(lam), L)
    fd = []
    for k in range(prob.Ns):
        e = np.zeros(prob.Ns)
        e[k] = H
        Xp, _, rp = O.pogm_unrolled(prob, NITER, list(lam * np.exp(e)), L)
        Xm, _, rm = O.pogm_unrolled(prob, NITER, list(lam * np.exp(-e)), L)
        assert rp == restarts and rm == restarts, "a restart decision moved within ±h"
        fd.append((O.unrolled_loss(Xp, Xt) - O.unrolled_loss(Xm, Xt)) / (2 * H))
    np.savez(OUT, loss=loss, grad=np.array(grad), fd=np.array(fd), h=H, lambdas=lam,
             restarts=np.array(restarts, dtype=np.uint8), niter=NITER, L=L)
    print("loss", loss, "grad", grad, "fd", fd)


if __name__ == "__main__":
    main()
