"""C-ABI checks that need no GPU: the library loads, exports every function
declared in include/mslr.h, and its host-only entry points (geometry,
argument validation) behave like the reference."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import mslr_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "mslr-recon_b200", "libmslr.so")
HDR = os.path.join(ROOT, "include", "mslr.h")


def declared_symbols():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"\b(mslr_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        pytest.fail("libmslr.so is not built (run __graft_entry__.build())")
    return C.CDLL(LIB)


def test_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_abi_version(lib):
    assert lib.mslr_abi_version() == 1


def _geom(lib, N, ps, ss):
    i3 = C.c_int32 * 3
    pso, nso = i3(), i3()
    Np = C.c_int64()
    rc = lib.mslr_patch_geometry(i3(*N), i3(*ps), i3(*ss), pso, nso, C.byref(Np), None)
    assert rc == 0
    st = (C.c_int32 * sum(v + 1 for v in nso))()
    rc = lib.mslr_patch_geometry(i3(*N), i3(*ps), i3(*ss), pso, nso, C.byref(Np), st)
    assert rc == 0
    return list(pso), list(nso), Np.value, list(st)


@pytest.mark.parametrize("seed", range(40))
def test_patch_geometry_bit_exact(lib, seed):
    rng = np.random.default_rng(seed)
    N = tuple(int(v) for v in rng.integers(1, 40, 3))
    ps = tuple(int(v) for v in rng.integers(1, 45, 3))
    ss = tuple(int(v) for v in rng.integers(1, 12, 3))
    ps_o, ns_o, Np, starts = _geom(lib, N, ps, ss)
    g = O.patch_geometry(N, ps, ss)
    assert tuple(ps_o) == g.ps
    assert tuple(ns_o) == g.nsteps
    assert Np == g.Np
    assert starts == [s for d in range(3) for s in g.starts[d]]


@pytest.mark.parametrize("N,ps,ss", [((90, 90, 60), (10, 10, 10), (5, 5, 5)),
                                     ((90, 90, 60), (6, 6, 6), (3, 3, 3)),
                                     ((32, 32, 24), (6, 6, 6), (6, 6, 6))])
def test_patch_geometry_workloads(lib, N, ps, ss):
    _, _, Np, starts = _geom(lib, N, ps, ss)
    g = O.patch_geometry(N, ps, ss)
    assert Np == g.Np
    assert starts == [s for d in range(3) for s in g.starts[d]]


def test_bad_arguments_rejected_without_gpu(lib):
    i3 = C.c_int32 * 3
    lib.mslr_last_error.restype = C.c_char_p
    h = C.c_void_p()
    # zero-size image: ArgumentError-equivalent, before any device work
    rc = lib.mslr_create(i3(0, 4, 4), 2, 3, C.c_int64(4), 1, i3(2, 2, 2), i3(2, 2, 2), 0, C.byref(h))
    assert rc == 1 and not h.value
    assert b"positive" in lib.mslr_last_error(None)
    # more samples than grid points
    rc = lib.mslr_create(i3(2, 2, 2), 2, 3, C.c_int64(9), 1, i3(2, 2, 2), i3(2, 2, 2), 0, C.byref(h))
    assert rc == 1
    # zero stride
    rc = lib.mslr_patch_geometry(i3(4, 4, 4), i3(2, 2, 2), i3(0, 1, 1), None, None, None, None)
    assert rc == 1
    # workspace query validates sizes
    b = C.c_size_t()
    assert lib.mslr_svst_batch_workspace(1000, 300, 486, C.byref(b)) == 0 and b.value > 0
    assert lib.mslr_svst_batch_workspace(2000, 2000, 1, C.byref(b)) == 4


def test_new_entries_reject_bad_arguments_without_gpu(lib):
    """The set-up, gradient, weight and tuning entries validate their
    arguments on the host (MSLR_ERR_ARG = 1) before any device work."""
    i3 = C.c_int32 * 3
    P = C.c_void_p
    K = C.c_int64()
    # null context
    assert lib.mslr_set_lambdas(None, (C.c_double * 2)(1.0, 2.0)) == 1
    assert lib.mslr_get_lambdas(None, (C.c_double * 2)()) == 1
    assert lib.mslr_autotune(None, None) == 1
    n = C.c_int32()
    assert lib.mslr_get_tuning(None, (C.c_int32 * 4)(), 4, C.byref(n)) == 1
    lib.mslr_pogm_grad.argtypes = [P, P, C.c_int32, C.c_double, C.c_double, C.c_double, P,
                                   P, P, P, P]
    assert lib.mslr_pogm_grad(None, None, 5, 2.0, 0.0, 1.0, None, None, None, None, None) == 1
    lib.mslr_prepare.argtypes = [P, P, P, P, P, P, P, P]
    assert lib.mslr_prepare(None, None, None, None, None, None, None, None) == 1
    # set-up entries: bad sizes and null pointers
    lib.mslr_sos_normalize.argtypes = [P, C.c_int32, P, P, P]
    assert lib.mslr_sos_normalize(i3(0, 4, 4), 2, P(16), P(16), None) == 1
    assert lib.mslr_sos_normalize(i3(4, 4, 4), 0, P(16), P(16), None) == 1
    assert lib.mslr_sos_normalize(i3(4, 4, 4), 2, None, P(16), None) == 1
    lib.mslr_sampling.argtypes = [P, C.c_int32, C.c_int32, P, P, P, P, C.c_int64, P]
    assert lib.mslr_sampling(i3(4, 4, 4), 2, 0, P(16), C.byref(K), None, None, 0, None) == 1
    assert lib.mslr_sampling(i3(4, 4, 4), 2, 3, None, C.byref(K), None, None, 0, None) == 1
    assert lib.mslr_sampling(i3(4, 4, 4), 2, 3, P(16), None, None, None, 0, None) == 1


def test_forms_are_declared():
    txt = open(HDR).read()
    for name, value in (("MSLR_FORM_PLAIN", 0), ("MSLR_FORM_TUNED", 1), ("MSLR_FORM_TF32", 2)):
        assert re.search(rf"#define {name} {value}\b", txt), name
