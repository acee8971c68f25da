#!/usr/bin/env python
"""POGM iterations/s of the MSLR hot path on B200.

Workload (the metric's configuration): N = (90, 90, 60) complex64, 18 coils,
Nt = 300, two scales — the global 90x90x60 patch and 10^3 patches with
stride 10 — on seeded synthetic data of those shapes (rank-8 temporal basis,
1/6 sampling with a 12^3 centre, normalised as run_recon does).  One step is
one POGM iteration: the SENSE normal operator, the fused u/z update with the
FP64 restart sums, and patch SVST over both scales.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU) runs independent replicas (weak
scaling); the value is the sum of iterations/s over ranks with the time
taken as the max over ranks.  ``--impl reference`` times the CPU port of the
reference algorithm (Julia is not available) on rank 0's host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "metric"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# each kernel of the SENSE chunk (6 coils x 4 frames at 90x90x60) from the ncu
# capture recorded in profiles/sense_four_pass_kernels_90x90x60.md; ncu
# flushes L2 before each launch, so these are cold-cache upper bounds (the
# timed loop finds most of the chunk's k-space in L2).
TRAFFIC_PER_LAUNCH = {"pfwd": 80505600, "zmask": 140111872, "padj": 162665984, "csum": 113441024}


def describe(pb) -> str:
    """Workload label, e.g. "90x90x60, 18 coils, Nt=300, scales [90,90,60]+[10,10,10] stride=size"."""
    Nt, Nc, _ = pb["y"].shape
    sc = "+".join("[%s]" % ",".join(str(v) for v in ps) for ps in pb["patch_sizes"])
    st = ("stride=size" if all(list(a) == list(b) for a, b in zip(pb["patch_sizes"], pb["strides"]))
          else "strides " + "+".join("[%s]" % ",".join(str(v) for v in ss) for ss in pb["strides"]))
    return f"{'x'.join(str(v) for v in pb['N'])}, {Nc} coils, Nt={Nt}, scales {sc} {st}"


METRIC = "POGM iter/s (90x90x60, 18 coils, Nt=300, 2 scales)"
# the bounded CPU sample, the same for cpu_baseline and the reference arm:
# fractions of the frames, of the local patches and of the global patch's rows
CPU_SAMPLE = (4 / 300, 12 / 486, 1 / 30)


def load_problem(name: str, seed_offset: int = 0):
    """Seeded synthetic problem of the named workload (the generator module is
    loaded by path so that the CPU-only reference arm needs no GPU library)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("mslr_synth_bench",
                                                  os.path.join(ROOT, "mslr-recon_b200", "synth.py"))
    S = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = S
    spec.loader.exec_module(S)
    import dataclasses
    cfg = dataclasses.replace(S.CONFIGS[name], seed=S.CONFIGS[name].seed + seed_offset)
    fft = "scipy"
    try:
        import torch
        if torch.cuda.is_available():
            fft = "torch"
    except Exception:
        pass
    t0 = time.perf_counter()
    pb = S.make_problem(cfg, fft=fft)
    log(f"generated {name} problem in {time.perf_counter() - t0:.1f}s ({fft} FFT)")
    return pb


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--form", default="tuned", choices=["tuned", "plain", "tf32"])
    p.add_argument("--workload", default=WORKLOAD)
    p.add_argument("--no-plain", action="store_true", help="skip the plain-form comparison")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--phases", action="store_true", help="print per-phase timings to stderr")
    p.add_argument("--files-recon", action="store_true",
                   help="with --workload files: also run run_recon_files on the written k-space (GPU)")
    return p.parse_args()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# clocks sampler
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU port (oracle restatement in FP32, all host threads) — bounded sample
# ---------------------------------------------------------------------------
def cpu_sample_iteration(pb, frac_frames: float, frac_patches: float, frac_rows: float, seed=0,
                         costs: dict | None = None):
    """Time a bounded sample of one POGM iteration of the CPU port and scale
    it to a full iteration.  Returns (seconds_per_iteration, description,
    threads).  With ``costs`` (a dict) it also times, on the same sample, the
    cost evaluations the reference's pogm_mod and logger add to every
    iteration — Fcost and the logger each run dc_cost (one forward SENSE) and
    reg_cost (svdvals of every patch of every scale) — and stores their
    scaled seconds per iteration under costs["seconds"]."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import mslr_oracle as O
    ncores = os.cpu_count() or 1
    smaps = pb["smaps"]
    idx = pb["idx"]
    y = pb["y"]
    Nt = y.shape[0]
    Nx, Ny, Nz = pb["N"]
    rng = np.random.default_rng(seed)
    x = pb["x_true"]
    # (a) data-consistency gradient on a subset of frames
    nf = max(1, int(round(frac_frames * Nt)))
    t0 = time.perf_counter()
    for t in range(nf):
        r = O.sense_forward_frame(x[t], smaps, idx[t], workers=ncores) - y[t]
        O.sense_adjoint_frame(r.astype(np.complex64), smaps, idx[t], workers=ncores)
    ta = (time.perf_counter() - t0) * Nt / nf
    # (b) local-scale SVST on a subset of patches (gesdd, thread pool)
    ps = pb["patch_sizes"][1]
    g = O.patch_geometry(pb["N"], ps, pb["strides"][1])
    npatch = max(1, int(round(frac_patches * g.Np)))
    mats = []
    for ip in rng.choice(g.Np, npatch, replace=False):
        sx, sy, sz = g.patch_start(int(ip))
        blk = x[:, sz:sz + ps[2], sy:sy + ps[1], sx:sx + ps[0]].reshape(Nt, -1).T.copy()
        mats.append(blk)
    lam = O.ong_lustig_lambdas(pb["N"], Nt, pb["patch_sizes"])
    from threadpoolctl import threadpool_limits
    t0 = time.perf_counter()
    with threadpool_limits(1, "blas"), ThreadPoolExecutor(ncores) as ex:   # one patch per thread
        list(ex.map(lambda m: O.svst(m, lam[1]), mats))
    tb = (time.perf_counter() - t0) * g.Np / npatch
    # (c) global patch: thin SVD cost is linear in rows — time a row subset
    nvox = Nx * Ny * Nz
    nrow = max(Nt, int(round(frac_rows * nvox)))
    G = x.reshape(Nt, nvox)[:, :nrow].T.copy()
    t0 = time.perf_counter()
    with threadpool_limits(ncores, "blas"):
        O.svst(G, lam[0])
    tc = (time.perf_counter() - t0) * nvox / nrow
    # (d) POGM elementwise on the same row subset, two scales
    xs = np.stack([x.reshape(Nt, nvox)[:, :nrow]] * 2)
    us = xs.copy()
    gg = x.reshape(Nt, nvox)[:, :nrow]
    t0 = time.perf_counter()
    un = xs - np.float32(0.5) * gg[None]
    zn = un + np.float32(0.3) * (un - us) + np.float32(0.6) * (un - xs)
    float(np.sum(np.real(-gg[None] * (un - us)), dtype=np.float64))
    td = (time.perf_counter() - t0) * nvox / nrow
    del zn
    if costs is not None:
        # dc_cost: A Σ_k X_k − y on the sampled frames; reg_cost: svdvals of the
        # sampled local patches and of the global patch's row subset; twice
        t0 = time.perf_counter()
        for t in range(nf):
            O.sense_forward_frame(x[t], smaps, idx[t], workers=ncores) - y[t]
        tfa = (time.perf_counter() - t0) * Nt / nf
        t0 = time.perf_counter()
        with threadpool_limits(1, "blas"), ThreadPoolExecutor(ncores) as ex:
            list(ex.map(lambda m: np.linalg.svd(m, compute_uv=False), mats))
        tfb = (time.perf_counter() - t0) * g.Np / npatch
        t0 = time.perf_counter()
        with threadpool_limits(ncores, "blas"):
            np.linalg.svd(G, compute_uv=False)
        tfc = (time.perf_counter() - t0) * nvox / nrow
        costs["seconds"] = 2.0 * (tfa + tfb + tfc)
    total = ta + tb + tc + td
    desc = (f"FP32 numpy/scipy port, {ncores} threads: normal op on {nf}/{Nt} frames, gesdd SVST on "
            f"{npatch}/{g.Np} 10^3 patches, global-patch SVD on {nrow}/{nvox} rows, POGM update on "
            f"the same rows; each scaled to one full iteration")
    return total, desc, ncores


def job_seconds(secs: float, world: int, dist=None, device=None) -> float:
    """Seconds of the whole job: the maximum of the ranks' timed seconds (the
    job ends when its slowest replica does).  Every rank gets the result."""
    if world <= 1:
        return secs
    import torch
    t = torch.tensor([secs], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world: int, steps: int, secs: float) -> float:
    """Whole-job iterations per second: every replica runs `steps` iterations."""
    return world * steps / secs


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    pb = load_problem(args.workload)
    secs = []
    desc = ""
    cores = 1
    for i in range(args.warmup + args.steps):
        s, desc, cores = cpu_sample_iteration(pb, *CPU_SAMPLE, seed=i)
        if i >= args.warmup:
            secs.append(s)
    v = 1.0 / (sum(secs) / len(secs))
    line = {"metric": METRIC, "value": v,
            "unit": "iter/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": describe(pb)},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "iter/s", "cores": cores, "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def time_steps(torch, ctx, X, steps, stream):
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        ctx.pogm_step(X, stream=stream)
    ev1.record(stream)
    ev1.synchronize()
    return ev0.elapsed_time(ev1) / 1000.0


def run_files(args):
    """The run_recon file path on the host: matwrite (deflate, all cores) and
    h5read of a zero-filled k-space ``ksp_epi_zf`` of the metric shape
    (90x90x60, 18 coils, Nt = 300, complex64, 21.0 GB; an 11^3 centre and
    1/6 of the voxels sampled in each frame, the same samples in every coil,
    seeded Gaussian values), through libmslrio.  Each step writes the file and reads
    it back; the file stays in the page cache.  The one-thread write and read
    and the pure-Python reader of the oracle run on a 20-frame file of the
    same kind; threads × the one-thread rate is the codec-bound ceiling the
    all-core figures are compared with."""
    import shutil
    import tempfile
    from mslr_recon_b200 import matio
    from oracle import h5_oracle
    Nt, Nc, (Nx, Ny, Nz) = 300, 18, (90, 90, 60)
    vox = Nx * Ny * Nz
    rng = np.random.default_rng(2024)
    ksp = np.zeros((Nt, Nc, vox), np.complex64)
    zc, yc, xc = np.meshgrid(np.arange(Nz) - Nz // 2, np.arange(Ny) - Ny // 2, np.arange(Nx) - Nx // 2,
                             indexing="ij")
    centre = ((np.abs(zc) < 6) & (np.abs(yc) < 6) & (np.abs(xc) < 6)).ravel()
    outer = np.flatnonzero(~centre)
    for t in range(Nt):       # the same sample count in every frame, as run_recon requires
        idx = np.union1d(np.flatnonzero(centre), rng.choice(outer, vox // 6, replace=False))
        ksp[t][:, idx] = (rng.standard_normal((Nc, idx.size), np.float32)
                          + 1j * rng.standard_normal((Nc, idx.size), np.float32))
    ksp = ksp.reshape(Nt, Nc, Nz, Ny, Nx)
    threads = os.cpu_count() or 1
    tmp = tempfile.mkdtemp(prefix="mslr_files_")
    try:
        path = os.path.join(tmp, "ksp.mat")
        steps = max(1, min(args.steps, 3))
        wr, rd = [], []
        for i in range(1 + steps):
            t0 = time.perf_counter()
            matio.matwrite(path, {"ksp_epi_zf": ksp}, compress=True, nthreads=threads)
            t1 = time.perf_counter()
            back = matio.h5read(path, "ksp_epi_zf", nthreads=threads)
            t2 = time.perf_counter()
            if i:
                wr.append(t1 - t0)
                rd.append(t2 - t1)
            ok = np.array_equal(back, ksp) if i == steps else True
            del back
            if not ok:
                raise RuntimeError("k-space read back differs from what was written")
        fbytes = os.path.getsize(path)
        recon = None
        if args.files_recon:
            from mslr_recon_b200.reconstruct import run_recon_files
            sm = (rng.standard_normal((Nc, Nz, Ny, Nx), np.float32)
                  + 1j * rng.standard_normal((Nc, Nz, Ny, Nx), np.float32)).astype(np.complex64)
            smaps_path = os.path.join(tmp, "smaps.mat")
            matio.matwrite(smaps_path, {"smaps": sm}, compress=True, nthreads=threads)
            niters = max(1, args.steps)
            fn_out, res = run_recon_files(path, smaps_path, os.path.join(tmp, "recon"), N=(Nx, Ny, Nz), Nvc=Nc,
                                          Nt=Nt, PATCH_SIZES=[[90, 90, 60], [10, 10, 10]],
                                          STRIDES=[[90, 90, 60], [10, 10, 10]], NITERS=niters,
                                          sigma1A_precomputed=1.0, nthreads=threads)
            recon = {"niters": niters, "seconds": res["seconds"], "out_file_gb": os.path.getsize(fn_out) / 1e9,
                     "note": "run_recon_files: h5read + matread, device set-up and POGM with cost logging "
                             "(sigma1 given), matwrite of the sixteen variables (deflate)"}
            del res
        small = os.path.join(tmp, "ksp20.mat")
        tw0 = time.perf_counter()
        matio.matwrite(small, {"ksp_epi_zf": ksp[:20]}, compress=True, nthreads=1)
        tw1 = time.perf_counter()
        t0 = time.perf_counter()
        one = matio.h5read(small, "ksp_epi_zf", nthreads=1)
        t1 = time.perf_counter()
        orc, _ = h5_oracle.OracleFile(small).read("/ksp_epi_zf")
        t2 = time.perf_counter()
        if not (np.array_equal(one, ksp[:20]) and np.array_equal(orc, ksp[:20])):
            raise RuntimeError("20-frame sample read back differs")
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    gb = ksp.nbytes / 1e9
    med_r, med_w = statistics.median(rd), statistics.median(wr)
    line = {"metric": "MAT v7.3 k-space read GB/s (ksp_epi_zf 90x90x60, 18 coils, Nt=300, c64, deflate)",
            "value": gb / med_r, "unit": "GB/s", "higher_is_better": True, "steps": steps, "warmup": 1,
            "dtype": "c64", "data": "synthetic",
            "config": {"workload": "zero-filled k-space 90x90x60x18x300 complex64, 11^3 centre + 1/6 of the voxels sampled per frame",
                       "array_gb": gb, "file_gb": fbytes / 1e9, "threads": threads,
                       "cache": "file in the host page cache"},
            "write_gbs": gb / med_w, "read_s": med_r, "write_s": med_w,
            "one_thread_read_gbs": ksp[:20].nbytes / 1e9 / (t1 - t0),
            "one_thread_write_gbs": ksp[:20].nbytes / 1e9 / (tw1 - tw0),
            "codec_roofline": {"read_frac": (gb / med_r) / (threads * ksp[:20].nbytes / 1e9 / (t1 - t0)),
                               "write_frac": (gb / med_w) / (threads * ksp[:20].nbytes / 1e9 / (tw1 - tw0)),
                               "note": "achieved over threads x the one-thread rate of the same codec path "
                                       "(zlib inflate / deflate bound)"},
            "cpu_baseline": {"value": ksp[:20].nbytes / 1e9 / (t2 - t1), "unit": "GB/s", "cores": 1,
                             "kind": "port", "sample": "pure-Python HDF5 reader (zlib inflate) on the "
                                                       "first 20 frames"}}
    if recon:
        line["run_recon_files"] = recon
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "files":
        return run_files(args)
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    import mslr_recon_b200 as M
    pb = load_problem(args.workload, seed_offset=rank)
    Nt, Nc, K = pb["y"].shape
    Nx, Ny, Nz = pb["N"]
    nvox = Nx * Ny * Nz
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    # host (pinned) inputs for the end-to-end leg
    h_smaps = torch.from_numpy(pb["smaps"]).pin_memory()
    h_y = torch.from_numpy(pb["y"]).pin_memory()
    h_idx = torch.from_numpy(pb["idx"]).pin_memory()
    L = float(len(pb["patch_sizes"]))   # σ1 = 1 (σ1A_PRECOMPUTED = 1.0 as the experiment files)

    def device_run(form, steps, warmup):
        ctx = M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form=form)
        ctx.bind(h_smaps.to(dev), h_y.to(dev), h_idx.to(dev))
        X = ctx.init_x0()
        ctx.pogm_begin(X, warmup + steps, L)
        for _ in range(warmup):
            ctx.pogm_step(X)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        n0 = ctx.launch_count()
        clocks = Clocks(local)
        clocks.start()
        secs = time_steps(torch, ctx, X, steps, stream)
        ck = clocks.stop()
        launches = ctx.launch_count() - n0
        torch.cuda.synchronize()
        secs = job_seconds(secs, world, dist, dev)
        return ctx, X, secs, ck, launches

    ctx, X, secs, clocks, launches = device_run(args.form, args.steps, args.warmup)
    tuning = ctx.tuning()
    value = job_value(world, args.steps, secs)

    # per-phase timing (same stream, CUDA events) for the roofline
    def ev_time(fn, reps=3):
        fn()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1000.0 / reps

    g = torch.empty((Nt, Nz, Ny, Nx), dtype=torch.complex64, device=dev)
    t_normal = ev_time(lambda: ctx.normal(X, out=g))
    tmp = torch.empty_like(g)
    t_svst = [ev_time(lambda k=k: ctx.patch_svst(k, 0.9 * ctx.lambdas[k], X[k], out=tmp))
              for k in range(ctx.Ns)]
    phases = {"normal_op_ms": t_normal * 1e3, "svst_ms": [t * 1e3 for t in t_svst]}
    if args.phases:
        log("phases", json.dumps(phases))
    # roofline: the dominant kernel of the iteration (the longest kernel of the
    # SENSE normal operator's chunks, per-launch device time from events around
    # every launch) and the whole iteration against Σ_steps max(bytes/BW, flops/peak)
    from mslr_recon_b200 import roofline as RL
    peaks = RL.peaks()
    fp32_tflops = M.fp32_peak()
    Ns = len(pb["patch_sizes"])
    roof = None
    try:
        kms, nl = ctx.normal_profile(X, out=g)
    except Exception as exc:   # shapes without the specialised kernels
        kms, nl = None, 0
        log("no per-kernel profile:", exc)
    ch = min(Nc, tuning["coils_per_group"])
    fr = tuning["frames_per_chunk"]
    if kms:
        phases["normal_op_kernel_ms"] = kms
        phases["normal_op_launches_per_kernel"] = nl
    if kms and "pfwd" in kms:
        per = RL.four_pass_kernels(pb["N"], ch, fr)
        names = {"pfwd": "k_pfwd (forward plane pass: coil map x summed image, DFT_y, DFT_x)",
                 "zmask": "k_zmask (z pass: DFT_z, k-space mask, inverse DFT_z)",
                 "padj": "k_padj (inverse plane pass: inverse DFT_y, DFT_x, x conj(coil map))",
                 "csum": "k_csum (coil combine into g)"}
        dom = max(("pfwd", "zmask", "padj"), key=lambda k: kms[k])
        tdom = kms[dom] / 1e3
        byts, fl = per[dom]["bytes"], per[dom]["flops"]
        achieved = byts / tdom / 1e9
        t_hbm, t_fp32 = byts / (peaks["hbm_gbs"] * 1e9), fl / (fp32_tflops * 1e12)
        roof = {"bound": "hbm", "kernel": names[dom],
                "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"],
                "traffic": TRAFFIC_PER_LAUNCH.get(dom),
                "algorithmic_bytes_per_launch": byts, "launch_ms": kms[dom],
                "peak_source": peaks["source"],
                "binding": "fp32" if t_fp32 > t_hbm else "hbm",
                "fp32": {"achieved_tflops": fl / tdom / 1e12, "peak_tflops": fp32_tflops,
                         "frac": fl / tdom / 1e12 / fp32_tflops,
                         "note": "nominal 5 N log2 N FFT flops per launch; peak measured by the "
                                 "library's FMA probe"},
                "kernels": {k: {"launch_ms": kms[k], "bytes": per[k]["bytes"], "flops": per[k]["flops"],
                                "hbm_frac": per[k]["bytes"] / (kms[k] / 1e3) / 1e9 / peaks["hbm_gbs"],
                                "fp32_frac": per[k]["flops"] / (kms[k] / 1e3) / 1e12 / fp32_tflops}
                            for k in per}}
    else:
        byts = RL.normal_op_bytes(nvox, Nt, Nc, Ns)
        achieved = byts / t_normal / 1e9
        roof = {"bound": "hbm", "kernel": "normal_op", "achieved": achieved, "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                "algorithmic_bytes": byts, "peak_source": peaks["source"]}
    scales = []
    for ps_, ss_ in zip(pb["patch_sizes"], pb["strides"]):
        gg = [min(a, b) for a, b in zip(ps_, pb["N"])]
        nst = [-(-(n - p_) // s_) + 1 for n, p_, s_ in zip(pb["N"], gg, ss_)]
        scales.append((gg[0] * gg[1] * gg[2], nst[0] * nst[1] * nst[2]))
    steps_ = RL.iteration_steps(pb["N"], Nt, Nc, scales)
    t_bound = RL.iteration_bound_seconds(steps_, peaks["hbm_gbs"], fp32_tflops, peaks["bf16_tflops_sustained"])
    t_iter = secs / args.steps
    roof["iteration_frac"] = t_bound / t_iter
    roof["iteration_bound_ms"] = t_bound * 1e3
    roof["iteration_note"] = ("sum over steps (normal operator, update, per scale the split-BF16 Gram/W/"
                              "rebuild products at a third of the sustained BF16 peak and the eigen stage "
                              "on the measured FP32 peak) of max(bytes/HBM, flops/peak), over the measured "
                              "iteration time")

    plain_ips = None
    plain_phases = None
    if not args.no_plain and args.form == "tuned":
        del ctx
        torch.cuda.empty_cache()
        psteps = max(2, args.steps // 2)
        pctx, pX, psecs, _, _ = device_run("plain", psteps, 1)
        plain_ips = world * psteps / psecs
        pg = torch.empty((Nt, Nz, Ny, Nx), dtype=torch.complex64, device=dev)
        pt_normal = ev_time(lambda: pctx.normal(pX, out=pg), reps=1)
        ptmp = torch.empty_like(pg)
        pt_svst = [ev_time(lambda k=k: pctx.patch_svst(k, 0.9 * pctx.lambdas[k], pX[k], out=ptmp), reps=1)
                   for k in range(pctx.Ns)]
        plain_ms = 1e3 * psecs / psteps
        plain_phases = {"iteration_ms": plain_ms, "normal_op_ms": pt_normal * 1e3,
                        "svst_ms": [t * 1e3 for t in pt_svst],
                        # the plain form with the tuned form's SENSE operator, from the two
                        # forms' measured phases: plain iteration − plain normal op + tuned normal op
                        "iteration_with_tuned_sense_ms": plain_ms - pt_normal * 1e3 + t_normal * 1e3}
        del pctx, pX, pg, ptmp
    else:
        del ctx
    torch.cuda.empty_cache()

    # end-to-end through the public API with host buffers (H2D + bind + POGM + D2H)
    e2e = None
    if not args.no_e2e:
        niter = args.steps
        h_out = torch.empty((Ns, Nt, Nz, Ny, Nx), dtype=torch.complex64).pin_memory()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d_s, d_y, d_i = (h_smaps.to(dev, non_blocking=True), h_y.to(dev, non_blocking=True),
                         h_idx.to(dev, non_blocking=True))
        ectx = M.MSLRContext(pb["N"], Nc, Nt, K, pb["patch_sizes"], pb["strides"], form=args.form)
        ectx.bind(d_s, d_y, d_i)
        EX = ectx.init_x0()
        ectx.pogm_run(EX, niter, L)
        h_out.copy_(EX, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        esecs = e0.elapsed_time(e1) / 1000.0
        if world > 1:
            t = torch.tensor([esecs], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            esecs = float(t.item())
        h2d = h_smaps.numel() * 8 + h_y.numel() * 8 + h_idx.numel() * 4
        d2h = h_out.numel() * 8
        e2e = {"value": world * niter / esecs, "unit": "iter/s",
               "h2d_bytes_per_step": h2d / niter, "d2h_bytes_per_step": d2h / niter,
               "note": f"one run_recon-style call of {niter} iterations per measurement; "
                       "inputs copied once per call, bytes shown per iteration"}
        ectx.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        extra = {}
        s, desc, cores = cpu_sample_iteration(pb, *CPU_SAMPLE, costs=extra)
        cpu = {"value": 1.0 / s, "unit": "iter/s", "cores": cores, "kind": "port", "sample": desc,
               "as_reference_iter_s": 1.0 / (s + extra["seconds"]),
               "as_reference_note": "with the per-iteration Fcost and logger cost evaluations the "
                                    "reference runs (2 forward SENSE passes and 2 svdvals sweeps)"}

    if world > 1:
        dist.barrier()
    if rank == 0:
        line = {"metric": METRIC, "value": value,
                "unit": "iter/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * secs / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
                "config": {"workload": describe(pb),
                           "form": args.form, "parallelism": f"replicas x{world}",
                           "tuning": tuning,
                           "l2": f"inputs larger than L2 (X is {pb['y'].shape[0] * nvox * 8 * len(pb['patch_sizes']) / 1e9:.1f} GB)",
                           "plain_form_iter_s": plain_ips,
                           "tuned_over_plain": (value / world / plain_ips * world) if plain_ips else None,
                           "tuned_over_plain_with_tuned_sense":
                               (plain_phases["iteration_with_tuned_sense_ms"] / (1e3 * secs / args.steps))
                               if plain_phases else None,
                           "phases": phases, "plain_phases": plain_phases},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
