"""Build libmslr.so (sm_100a) in-tree with nvcc.

Usage: ``python mslr-recon_b200/build_lib.py [--force] [--verbose]``.
Objects go to ``_build/`` at the repository root; the shared library is
written next to this file so that it travels with the package.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libmslr.so")
IO_LIB = os.path.join(HERE, "libmslrio.so")
IO_SRC = os.path.join(CSRC, "matio.cpp")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O3", "-Xptxas", "-O3", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "mslr.h"))
    return hs


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    """Compile every .cu under csrc/ and link libmslr.so; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    exe = nvcc()
    hdrs = headers()
    flags = NVCC_FLAGS + list(extra_flags or [])
    objs, jobs = [], []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            cmd = [exe, *ARCH, *flags, "-I", CSRC, "-I", os.path.join(ROOT, "include"),
                   "-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {cmd[-3]}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, flush=True)
        return r

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or _stale(LIB, objs):
        cmd = [exe, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def build_io(force: bool = False, verbose: bool = False) -> str:
    """Compile the host-only MAT v7.3 / HDF5 library libmslrio.so (g++, zlib)."""
    hdr = os.path.join(ROOT, "include", "mslr_io.h")
    if force or _stale(IO_LIB, [IO_SRC, hdr]):
        cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
        cmd = [cxx, "-std=c++17", "-O3", "-fPIC", "-shared", "-Wall", "-I", os.path.join(ROOT, "include"),
               IO_SRC, "-o", IO_LIB, "-lz", "-pthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed for matio.cpp:\n{r.stdout}\n{r.stderr}")
    return IO_LIB


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(p)
    print(build_io(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
