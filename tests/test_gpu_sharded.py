"""The sharded iteration (mslr-recon_b200/sharded.py) end to end on the GPU:
two ranks run as two processes on the one GPU, their collectives through
gloo on the host (no kernel of one rank waits on the other's).  Frames
[0, 8) and [8, 16) of a 32×32×24, 8-coil, Nt = 16 problem go to ranks 0 and
1 for the SENSE operator; z-slabs [0, 16) and [16, 24) for the SVST of the
global patch (partial Grams all-reduced) and of the 8³ patches.  Each rank's
frames of X after every iteration are compared with the FP64 oracle, and
the restart flags must agree with it on both ranks."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NITER = 4


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    import dataclasses
    import sys
    from tests.conftest import load_synth
    synth = load_synth()
    cfg = dataclasses.replace(synth.CONFIGS["small"], Nt=16, patch_sizes=[[32, 32, 24], [8, 8, 8]],
                              strides=[[32, 32, 24], [8, 8, 8]])
    return synth.make_problem(cfg)


def _worker(rank, world, port, out_dir, form):
    import datetime
    import sys

    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle import mslr_oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    import mslr_recon_b200.sharded as S
    pb = _problem()
    Nt, Nc, K = pb["y"].shape
    prob = O.ReconProblem(smaps=pb["smaps"].astype(np.complex128), idx=pb["idx"],
                          y=pb["y"].astype(np.complex128), patch_sizes=pb["patch_sizes"],
                          strides=pb["strides"], sigma1=1.0)
    traj = []
    _, restarts, _, _ = O.run_recon_arrays(prob, NITER, iter_callback=lambda it, xk, r: traj.append(xk.copy()))
    sh = S.ShardedRecon(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form=form)
    t0, t1 = sh.frames[rank]
    sh.bind(torch.from_numpy(pb["smaps"]).cuda(), torch.from_numpy(pb["y"][t0:t1].copy()).cuda(),
            torch.from_numpy(pb["idx"][t0:t1].copy()).to(torch.int32).cuda())
    errs = []
    flags = sh.run(NITER, float(len(pb["patch_sizes"])),
                   callback=lambda it, Xf: errs.append(O.rel_err(Xf.cpu().numpy(), traj[it - 1][:, t0:t1])))
    sh.close()
    with open(os.path.join(out_dir, f"r{rank}"), "w") as f:
        f.write(" ".join(f"{e:.3e}" for e in errs) + "\n")
        f.write("same" if flags == restarts else f"flags {flags} vs {restarts}")
    dist.destroy_process_group()


@pytest.mark.parametrize("form", ["tuned", "plain"])
def test_sharded_iteration_two_ranks_matches_oracle(tmp_path, form):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), form), nprocs=2, join=True)
    for r in range(2):
        errs, flags = (tmp_path / f"r{r}").read_text().split("\n")
        print(f"{form} rank {r}: per-iteration rel err {errs}")
        assert flags == "same", flags
        assert max(float(v) for v in errs.split()) < 1e-4, errs
