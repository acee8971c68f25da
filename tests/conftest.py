"""Shared test setup: import paths, the ``gpu`` marker and small fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The oracle runs many small LAPACK calls (one SVD per patch); a multithreaded
# BLAS spends more time synchronising than computing on them.
try:
    from threadpoolctl import threadpool_limits
    threadpool_limits(1, "blas")
except Exception:
    pass


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libmslr.so")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def load_synth():
    """The package's synthetic generator, loaded without the package (so the
    CPU tests do not need libmslr.so)."""
    import importlib.util
    name = "mslr_synth_standalone"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "mslr-recon_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def synth():
    return load_synth()


@pytest.fixture(scope="session")
def small_problem(synth):
    """The small CPU-runnable workload (32x32x24, 8 coils, Nt=64, rank 4)."""
    return synth.make_problem(synth.CONFIGS["small"])


def rng(seed=0):
    return np.random.default_rng(seed)
