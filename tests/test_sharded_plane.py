"""Data plane of the sharded iteration (mslr-recon_b200/sharded.py) on CPU:
the frame / slab partition and the all-to-all moves between frame layout
and slab layout, with two gloo ranks (no GPU needed)."""
import os
import socket

import pytest
import torch

from tests.conftest import ROOT  # noqa: F401  (import path)


def _sharded():
    import importlib.util
    import sys
    sys.path.insert(0, ROOT)
    import mslr_recon_b200.sharded as S
    return S


def test_split_range_and_slab_unit():
    S = _sharded()
    assert S.split_range(300, 2) == [(0, 150), (150, 300)]
    assert S.split_range(60, 4, 10) == [(0, 20), (20, 40), (40, 50), (50, 60)]
    assert S.split_range(7, 3) == [(0, 3), (3, 5), (5, 7)]
    with pytest.raises(ValueError):
        S.split_range(60, 7, 10)   # six z patch rows cannot feed seven ranks
    assert S.slab_unit((90, 90, 60), [[90, 90, 60], [10, 10, 10]], [[90, 90, 60], [10, 10, 10]]) == 10
    assert S.slab_unit((32, 32, 24), [[32, 32, 24], [8, 8, 8], [4, 4, 6]],
                       [[32, 32, 24], [8, 8, 8], [4, 4, 6]]) == 24
    with pytest.raises(ValueError):   # half-overlapping patches need halos
        S.slab_unit((90, 90, 60), [[90, 90, 60], [10, 10, 10]], [[90, 90, 60], [5, 5, 5]])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    S = _sharded()
    Ns, Nt, Nz, Ny, Nx = 2, 7, 12, 3, 4
    g = torch.Generator().manual_seed(5)
    full = torch.complex(torch.randn(Ns, Nt, Nz, Ny, Nx, generator=g), torch.randn(Ns, Nt, Nz, Ny, Nx, generator=g))
    frames = S.split_range(Nt, world)
    slabs = S.split_range(Nz, world, 3)
    t0, t1 = frames[rank]
    z0, z1 = slabs[rank]
    Zf = full[:, t0:t1].contiguous()
    Zs = torch.empty((Ns, Nt, z1 - z0, Ny, Nx), dtype=torch.complex64)
    S.frames_to_slabs(Zf, frames, slabs, rank, Zs)
    ok1 = torch.equal(Zs, full[:, :, z0:z1])
    back = torch.empty_like(Zf)
    S.slabs_to_frames(Zs, frames, slabs, rank, back)
    ok2 = torch.equal(back, Zf)
    s = torch.full((4,), float(rank + 1), dtype=torch.float64)
    S._sum_over_ranks(s)
    ok3 = bool(torch.all(s == sum(range(1, world + 1))))
    with open(os.path.join(out_dir, f"r{rank}"), "w") as f:
        f.write(f"{int(ok1)}{int(ok2)}{int(ok3)}")
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_frames_slabs_all_to_all_round_trip(tmp_path, world):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        assert (tmp_path / f"r{r}").read_text() == "111", r
