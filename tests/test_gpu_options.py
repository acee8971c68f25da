"""pogm_mod's other options through ``mslr_pogm_run_options``.

run_recon calls pogm_mod with mom = :pogm, restart = :gr and f_mu = 0
(scripts/reconstruct.jl:217); pogm_mod itself (src/mirt_mod.jl:74-188) also
offers mom = :pgm / :fpgm, restart = :none / :fr and a strong-convexity
parameter f_mu > 0.  Each combination below runs on the GPU from X0 = A'y
and is compared with the FP64 oracle's restatement of pogm_mod driven by the
same closures: the returned iterate (xnew for :pogm, ynew otherwise) and the
restart flags.  :fr uses run_recon's comp_cost = dc_cost + reg_cost.
"""
import dataclasses

import numpy as np
import pytest

from oracle import mslr_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-4

# (mom, restart, f_mu, restart_cutoff, bsig, sigma1, niter, form).  L = Ns·sigma1²;
# sigma1 < 1 overstates the step (the coil maps give a true σ1 of 1), so the
# cost rises in some iterations and the function restart fires; the chosen
# settings mix restarted and non-restarted iterations, with the cost change at
# every :fr decision at least 0.4 % of the cost (FP32 costs agree to ~1e-6)
# and the cosine of every :gr decision at least 1e-4 from the cutoff.
CASES = [
    ("pgm", "none", 0.0, 0.0, 1.0, 1.0, 8, "tuned"),
    ("pgm", "gr", 0.0, 0.1, 1.0, 1.0, 8, "tuned"),      # restarts every iteration
    ("pgm", "fr", 0.0, 0.0, 1.0, 0.65, 12, "plain"),    # restarts at 11, 12
    ("pgm", "gr", 0.3, 0.0, 1.0, 1.0, 8, "tuned"),
    ("fpgm", "none", 0.0, 0.0, 1.0, 1.0, 8, "tuned"),
    ("fpgm", "gr", 0.0, 0.0018, 1.0, 1.0, 12, "tuned"), # restarts at 1, 2
    ("fpgm", "gr", 0.0, 0.0, 1.0, 1.0, 8, "plain"),
    ("fpgm", "fr", 0.0, 0.0, 1.0, 0.75, 12, "tuned"),   # restart at 11
    ("fpgm", "gr", 0.3, 0.0, 1.0, 1.0, 8, "tuned"),
    ("pogm", "none", 0.0, 0.0, 1.0, 1.0, 8, "tuned"),
    ("pogm", "fr", 0.0, 0.0, 0.8, 0.85, 16, "tuned"),   # restarts at 6, 8-15; σ decreases
    ("pogm", "fr", 0.0, 0.0, 1.0, 0.85, 12, "plain"),
    ("pogm", "gr", 0.3, 0.0, 1.0, 1.0, 8, "tuned"),
    ("pogm", "gr", 0.3, 0.1, 0.8, 1.0, 8, "plain"),
    ("pogm", "gr", 0.0, 0.003, 0.8, 1.0, 12, "tuned"),  # run_recon's choice (mslr_pogm_run); 1-5
]


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
def problem(synth):
    cfg = dataclasses.replace(synth.CONFIGS["small"], Nt=16)
    return synth.make_problem(cfg)


def _oracle_problem(pb, sigma1=1.0):
    return O.ReconProblem(smaps=pb["smaps"].astype(np.complex128), idx=pb["idx"],
                          y=pb["y"].astype(np.complex128), patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"], sigma1=sigma1)


@pytest.mark.parametrize("mom,restart,f_mu,cutoff,bsig,sigma1,niter,form", CASES)
def test_pogm_options_match_oracle(torch, M, problem, mom, restart, f_mu, cutoff, bsig, sigma1, niter,
                                   form):
    pb = problem
    Nt, Nc, K = pb["y"].shape
    prob = _oracle_problem(pb, sigma1)
    L = prob.lipschitz()
    Xo, restarts, _, _ = O.run_recon_arrays(prob, niter, mom=mom, restart=restart, f_mu=f_mu,
                                            restart_cutoff=cutoff, bsig=bsig)
    with M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form=form) as ctx:
        ctx.bind(torch.from_numpy(pb["smaps"]).cuda(), torch.from_numpy(pb["y"]).cuda(),
                 torch.from_numpy(pb["idx"]).to(torch.int32).cuda())
        X = ctx.init_x0()
        flags = ctx.pogm_run_options(X, niter, L, mom=mom, restart=restart, f_mu=f_mu,
                                     restart_cutoff=cutoff, bsig=bsig)
        err = O.rel_err(X.cpu().numpy(), Xo)
    print(f"{mom}/{restart}/mu={f_mu}/cutoff={cutoff}/bsig={bsig}/L={L:.3f}/{form}: rel err {err:.2e}, "
          f"restarts {[i for i, v in enumerate(flags) if v]}")
    assert err < TOL
    assert flags == restarts


def test_pogm_options_argument_errors(torch, M, problem):
    """pogm_mod's ArgumentErrors (src/mirt_mod.jl:88-93) as MSLR_ERR_ARG."""
    from mslr_recon_b200._lib import MSLR_ERR_ARG, lib
    pb = problem
    Nt, Nc, K = pb["y"].shape
    with M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"]) as ctx:
        ctx.bind(torch.from_numpy(pb["smaps"]).cuda(), torch.from_numpy(pb["y"]).cuda(),
                 torch.from_numpy(pb["idx"]).to(torch.int32).cuda())
        X = ctx.init_x0()
        with pytest.raises(ValueError):
            ctx.pogm_run_options(X, 2, 2.0, mom="gd")
        with pytest.raises(ValueError):
            ctx.pogm_run_options(X, 2, 2.0, restart="always")
        for args in [(2, 2.0, 0.0, 3, 1, 0.0, 1.0),     # mom out of range
                     (2, 2.0, 0.0, 2, 5, 0.0, 1.0),     # restart out of range
                     (2, 2.0, -1.0, 2, 1, 0.0, 1.0),    # f_mu < 0
                     (2, 2.0, 0.0, 2, 1, 1.0, 1.0),     # |restart_cutoff| >= 1
                     (2, 2.0, 0.0, 2, 1, 0.0, -0.5)]:   # bsig < 0
            rc = lib.mslr_pogm_run_options(ctx._h, X.data_ptr(), *args, None, None)
            assert rc == MSLR_ERR_ARG, args
        with pytest.raises(ValueError):   # MSLR_ERR_ARG is raised as ValueError
            ctx.pogm_run_options(X, 2, 2.0, f_mu=-1.0)
