"""The N > 1 path of bench.py (one replica per GPU, no collective on the data
path) on the CPU: two gloo ranks agree on the whole job's time — the maximum
of their timed seconds — and on the job's throughput, and under torchrun only
rank 0 runs the reference arm."""
import importlib.util
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def load_bench():
    spec = importlib.util.spec_from_file_location("mslr_bench_mr", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench = load_bench()
        secs = 1.0 + 0.5 * rank            # rank 1 is the slower replica
        job = bench.job_seconds(secs, world, dist)
        q.put((rank, job, bench.job_value(world, 10, job)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, job, value in got:
        assert job == pytest.approx(1.5)
        assert value == pytest.approx(2 * 10 / 1.5)


def test_single_rank_is_its_own_job():
    bench = load_bench()
    assert bench.job_seconds(2.5, 1) == 2.5
    assert bench.job_value(1, 10, 2.5) == pytest.approx(4.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    bench = load_bench()
    monkeypatch.setenv("RANK", "1")
    import argparse
    ns = argparse.Namespace(workload="small", warmup=0, steps=1, gpus=2)
    assert bench.run_reference(ns) == 0
    assert capsys.readouterr().out == ""
