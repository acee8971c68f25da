"""MAT v7.3 / HDF5 reader and writer (libmslrio.so), on the CPU.

The reference reads its coil maps and k-space through MAT.jl / HDF5.jl and
saves its results through MAT.jl (scripts/reconstruct.jl:88,95,242-260).
Neither Julia nor libhdf5 is in this image, so the checks are:

- the pin: a MATLAB-written v7.3 file from scipy's test data
  (``testhdf5_7.4_GLNX86.mat``, ``testdouble`` = 0:pi/4:2*pi, written by
  MATLAB's libhdf5) read bit-exactly by the library and by the independent
  pure-Python reader ``oracle/h5_oracle.py``; the same variable from its
  MATLAB v5 twin (read by scipy.io.loadmat) agrees;
- every file the library writes is decoded identically by the oracle reader
  (a second implementation of the format), bit-exact;
- files in the newer HDF5 structures the writer does not produce
  (superblock 2, object header 2, link messages, layout 4 with single-chunk,
  implicit and fixed-array chunk indexes, filter pipeline 2 with shuffle,
  attribute 3, compact layout) are assembled here byte by byte from the
  format specification and read back bit-exactly;
- damaged and foreign files fail with a status, never a crash.
"""
import os
import zlib

import numpy as np
import pytest

from oracle import h5_oracle as H

matio = pytest.importorskip("mslr_recon_b200.matio")

SCIPY_DATA = os.path.join(os.path.dirname(__import__("scipy").__file__), "io", "matlab", "tests", "data")
MATLAB_V73 = os.path.join(SCIPY_DATA, "testhdf5_7.4_GLNX86.mat")
MATLAB_V5 = os.path.join(SCIPY_DATA, "testdouble_7.4_GLNX86.mat")


# ───────────────────────── the pin: a MATLAB-written file ─────────────────────────

@pytest.mark.skipif(not os.path.exists(MATLAB_V73), reason="scipy test data not installed")
def test_matlab_written_file_bit_exact():
    want = np.arange(9) * (np.pi / 4)
    with matio.H5File(MATLAB_V73) as f:
        assert f.userblock == 512
        assert f.names() == ["testdouble"]
        inf = f.info("/testdouble")
        assert inf.shape == (9, 1) and inf.mclass == "double" and inf.layout == 1
        a = f.read_raw("/testdouble")
    assert np.array_equal(a.ravel(), want)            # bit-exact: MATLAB stored 0:pi/4:2*pi
    o = H.OracleFile(MATLAB_V73)
    b, attrs = o.read("/testdouble")
    assert np.array_equal(a, b) and attrs["MATLAB_class"] == "double"
    text, ver, endian = H.matlab_header(MATLAB_V73)
    assert text.startswith("MATLAB 7.0 MAT-file") and ver == b"\x00\x02" and endian == b"IM"
    assert matio.matread(MATLAB_V73)["testdouble"].shape == (9, 1)


@pytest.mark.skipif(not (os.path.exists(MATLAB_V73) and os.path.exists(MATLAB_V5)),
                    reason="scipy test data not installed")
def test_v73_and_v5_files_agree():
    a = matio.matread(MATLAB_V73)["testdouble"]
    b = matio.matread(MATLAB_V5)["testdouble"]
    assert a.shape == b.shape and np.array_equal(a, b)


def test_v5_files_use_the_same_dims_convention(tmp_path):
    """Coil maps saved by MATLAB without -v7.3 are MAT v5 files (read through
    scipy.io.loadmat); they come back in the reversed-dims convention of the
    v7.3 reader, so both kinds feed run_recon_files alike."""
    from scipy.io import savemat
    rng = np.random.default_rng(23)
    sm = (rng.standard_normal((5, 4, 3, 2)) + 1j * rng.standard_normal((5, 4, 3, 2))).astype(np.complex64)
    # a MATLAB array of size (Nx, Ny, Nz, Nc) = (5, 4, 3, 2), column-major
    p5, p73 = str(tmp_path / "smaps_v5.mat"), str(tmp_path / "smaps_v73.mat")
    savemat(p5, {"smaps": np.asfortranarray(sm), "R": 2.5})
    matio.matwrite(p73, {"smaps": np.ascontiguousarray(sm.T), "R": 2.5})
    a, b = matio.matread(p5), matio.matread(p73)
    assert a["smaps"].shape == b["smaps"].shape == (2, 3, 4, 5)
    assert np.array_equal(a["smaps"], b["smaps"]) and np.array_equal(a["smaps"], sm.T)
    assert a["R"] == b["R"] == 2.5


# ───────────────────────── writer ↔ reader ↔ oracle ─────────────────────────

def _variables(rng):
    c = (rng.standard_normal((3, 5, 7, 9)) + 1j * rng.standard_normal((3, 5, 7, 9))).astype(np.complex64)
    return {
        "X": c,
        "Xd": c.astype(np.complex128)[:, :2],
        "f32": rng.standard_normal((11, 13)).astype(np.float32),
        "f64": rng.standard_normal((4, 1, 6)),
        "vec": rng.standard_normal(10),
        "i8": rng.integers(-128, 127, (5, 3), dtype=np.int8),
        "u16": rng.integers(0, 65535, (7,), dtype=np.uint16),
        "i32": rng.integers(-2**31, 2**31 - 1, (2, 3, 4), dtype=np.int32),
        "u32": rng.integers(0, 2**32 - 1, (6, 2), dtype=np.uint32),
        "i64": rng.integers(-2**62, 2**62, (3, 3), dtype=np.int64),
        "u64": rng.integers(0, 2**63, (2, 5), dtype=np.uint64),
        "mask": rng.random((4, 6, 5)) > 0.5,
        "scalar_f": 2.5,
        "scalar_i": 7,
        "flag": True,
        "text": "run_recon ✓ 𝛌",
        "cells": [np.arange(3, dtype=np.int64), np.arange(4.0), "ab"],
        "empty": np.zeros((0, 3)),
        "r6": rng.standard_normal((2, 3, 1, 2, 3, 2)).astype(np.float32),
    }


def _as_written(v):
    """What matread returns for a value matwrite was given."""
    if isinstance(v, np.ndarray) and v.ndim == 1:
        return v.reshape(1, -1)
    return v


def _equal(a, b):
    if isinstance(a, list):
        return isinstance(b, list) and len(a) == len(b) and all(_equal(_as_written(x), y) for x, y in zip(a, b))
    if isinstance(a, np.ndarray):
        return isinstance(b, np.ndarray) and a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a, b)
    return type(a) is type(b) and a == b


@pytest.mark.parametrize("compress,chunk", [(False, 0), (True, 4 << 20), (True, 64), (True, 24)])
def test_round_trip_every_type(tmp_path, compress, chunk):
    rng = np.random.default_rng(7)
    d = _variables(rng)
    p = str(tmp_path / "v.mat")
    matio.matwrite(p, d, compress=compress, chunk_bytes=chunk or (4 << 20))
    r = matio.matread(p)
    assert set(r) == set(d)
    for k, v in d.items():
        assert _equal(_as_written(v), r[k]), k


@pytest.mark.parametrize("chunk", [0, 96, 4 << 20])
def test_oracle_reads_what_the_library_writes(tmp_path, chunk):
    rng = np.random.default_rng(11)
    d = {k: v for k, v in _variables(rng).items() if isinstance(v, np.ndarray) and v.size and v.dtype != np.bool_}
    p = str(tmp_path / "o.mat")
    matio.matwrite(p, d, compress=chunk > 0, chunk_bytes=chunk or (4 << 20))
    o = H.OracleFile(p)
    assert o.base_field == 512 and o.sb == 512
    assert o.eof_field == os.path.getsize(p)
    text, ver, endian = H.matlab_header(p)
    assert text.startswith("MATLAB 7.3 MAT-file") and ver == b"\x00\x02" and endian == b"IM"
    names = sorted(n for n, _ in o.members(o.root))
    assert names == sorted(d)
    with matio.H5File(p) as f:
        for k, v in d.items():
            a, attrs = o.read("/" + k)
            assert np.array_equal(a, _as_written(v)), k
            assert a.dtype == v.dtype
            assert np.array_equal(f.read_raw("/" + k), a), k
            assert attrs["MATLAB_class"] == f.info("/" + k).mclass


def test_writer_follows_libhdf5_layout_rules(tmp_path):
    """The structures libhdf5 itself checks or sizes from the superblock:
    message counts (the oracle checks every header it parses), full-size
    symbol and B-tree nodes, names sorted and bracketed by the group
    B-tree's keys, the heap's free-list sentinel, chunk keys in order with
    the right-most key one chunk past the last, exact contiguous sizes."""
    rng = np.random.default_rng(13)
    a = rng.standard_normal((7, 9, 5)).astype(np.float32)
    d = {"zeta": a, "alpha": np.arange(10.0), "cell": [np.arange(2), np.arange(3.0)], "mid": 3}
    p = str(tmp_path / "rules.mat")
    matio.matwrite(p, d, compress=True, chunk_bytes=5 * 4 * 2)     # chunks of (1, 2, 5): 7 x 5 = 35 of them
    o = H.OracleFile(p)
    b, so = o.b, o.so
    assert o.internal_k == 16 and o.leaf_k >= 4

    def u(x, n=8):
        return int.from_bytes(b[x:x + n], "little")

    for group in ("/", "/#refs#"):
        msgs = o.messages(o.lookup(group))
        stab = [m for t, _, m in msgs if t == 0x11][0]
        bt, heap = int.from_bytes(stab[:8], "little"), int.from_bytes(stab[8:16], "little")
        h = o.abs(heap)
        assert b[h:h + 4] == b"HEAP" and u(h + 16) == 1                  # free list: none
        dseg, dsize = o.abs(u(h + 24)), u(h + 8)
        assert dsize % 8 == 0
        n = o.abs(bt)
        assert b[n:n + 4] == b"TREE" and b[n + 4] == 0 and b[n + 5] == 0 and u(n + 6, 2) == 1
        assert n + 24 + 33 * 8 + 32 * 8 <= len(b)                         # full node of 2K = 32 children
        k0, child, k1 = u(n + 24), u(n + 32), u(n + 40)
        names = [nm for nm, _ in o.members(o.lookup(group))]
        assert names == sorted(names, key=lambda x: x.encode())
        name_at = lambda off: b[dseg + off:b.index(b"\0", dseg + off)].decode()
        assert name_at(k0) == "" and name_at(k1) == names[-1]
        sn = o.abs(child)
        assert b[sn:sn + 4] == b"SNOD" and u(sn + 6, 2) == len(names)
        assert sn + 8 + 2 * o.leaf_k * 40 <= len(b)                      # full node of 2·leaf K entries

    msgs = dict((t, m) for t, _, m in o.messages(o.lookup("/zeta")))
    lay = msgs[0x08]
    assert lay[0] == 3 and lay[1] == 2 and lay[2] == 4
    cd = [int.from_bytes(lay[11 + 4 * i:15 + 4 * i], "little") for i in range(4)]
    assert cd == [1, 2, 5, 4]
    n = o.abs(int.from_bytes(lay[3:11], "little"))
    assert b[n + 4] == 1 and b[n + 5] == 0 and u(n + 6, 2) == 35       # 35 chunks fit one leaf
    ks = 8 + 8 * 4
    keys = [tuple(u(n + 24 + i * (ks + so) + 8 + 8 * j) for j in range(4)) for i in range(36)]
    assert keys[:-1] == sorted(keys[:-1]) and len(set(keys[:-1])) == 35
    assert keys[-1] == (keys[-2][0] + 1, keys[-2][1] + 2, keys[-2][2] + 5, 4)
    assert n + 24 + 65 * ks + 64 * so <= len(b)                           # full node of 2K = 64 children

    p2 = str(tmp_path / "contig.mat")
    matio.matwrite(p2, {"alpha": np.arange(10.0)})
    o2 = H.OracleFile(p2)
    msgs = dict((t, m) for t, _, m in o2.messages(o2.lookup("/alpha")))
    assert msgs[0x08][:2] == bytes([3, 1]) and int.from_bytes(msgs[0x08][10:18], "little") == 80


def test_many_chunks_multilevel_btree(tmp_path):
    # 5000 chunks of one row each: three B-tree levels with 64 entries per node
    rng = np.random.default_rng(3)
    a = rng.standard_normal((5000, 3)).astype(np.float32)
    p = str(tmp_path / "m.mat")
    matio.matwrite(p, {"a": a}, compress=True, chunk_bytes=12)
    with matio.H5File(p) as f:
        inf = f.info("/a")
        assert inf.layout == 2 and inf.chunk[0] == 1 and inf.n_filters == 1
        for t in (1, 3, 8):
            f.nthreads = t
            assert np.array_equal(f.read_raw("/a"), a)
    b, _ = H.OracleFile(p).read("/a")
    assert np.array_equal(b, a)


def test_edge_chunks_and_incompressible_chunks(tmp_path):
    rng = np.random.default_rng(5)
    noise = rng.integers(0, 256, (37, 29, 3), dtype=np.uint8)       # does not compress: stored raw
    zeros = np.zeros((37, 29, 3), dtype=np.uint8)                   # compresses
    p = str(tmp_path / "e.mat")
    matio.matwrite(p, {"noise": noise, "zeros": zeros}, compress=True, chunk_bytes=1000)
    o = H.OracleFile(p)
    for k, v in (("noise", noise), ("zeros", zeros)):
        a, _ = o.read("/" + k)
        assert np.array_equal(a, v)
        assert np.array_equal(matio.h5read(p, k), v)
    assert os.path.getsize(p) < noise.nbytes + 64 * 1024


def test_large_complex_array_threads(tmp_path):
    rng = np.random.default_rng(9)
    x = (rng.standard_normal((6, 4, 30, 40, 50)) + 1j * rng.standard_normal((6, 4, 30, 40, 50))).astype(np.complex64)
    p = str(tmp_path / "k.mat")
    matio.matwrite(p, {"ksp_epi_zf": x}, compress=True, nthreads=8, chunk_bytes=1 << 18)
    for t in (1, 8):
        assert np.array_equal(matio.h5read(p, "ksp_epi_zf", nthreads=t), x)


# ───────────────────────── newer HDF5 structures, assembled here ─────────────────────────

def _u(v, n):
    return int(v).to_bytes(n, "little")


def _dt_float(size):
    if size == 4:
        props = _u(0, 2) + _u(32, 2) + bytes([23, 8, 0, 23]) + _u(127, 4)
    else:
        props = _u(0, 2) + _u(64, 2) + bytes([52, 11, 0, 52]) + _u(1023, 4)
    return bytes([0x11, 0x20, 31 if size == 4 else 63, 0]) + _u(size, 4) + props


def _dt_complex3(size):
    """Compound datatype version 3 (packed member names, minimal offsets)."""
    fs = size // 2
    body = b""
    for i, nm in enumerate((b"r", b"i")):
        body += nm + b"\0" + _u(i * fs, 1) + _dt_float(fs)
    return bytes([0x36, 2, 0, 0]) + _u(size, 4) + body


def _space2(dims):
    return bytes([2, len(dims), 0, 1]) + b"".join(_u(d, 8) for d in dims)


def _attr3(name, value: bytes):
    dt = bytes([0x13, 0, 0, 0]) + _u(len(value), 4)
    sp = bytes([2, 0, 0, 0])
    nm = name.encode() + b"\0"
    return bytes([3, 0]) + _u(len(nm), 2) + _u(len(dt), 2) + _u(len(sp), 2) + b"\0" + nm + dt + sp + value


class _V2File:
    """Superblock 2, version-2 object headers, link messages (checksums are
    written as zeros: the library does not verify them)."""

    def __init__(self):
        self.buf = bytearray(48)

    def alloc(self, data: bytes) -> int:
        a = len(self.buf)
        self.buf += data
        while len(self.buf) % 8:
            self.buf.append(0)
        return a

    @staticmethod
    def ohdr(msgs):
        body = b"".join(bytes([t]) + _u(len(d), 2) + b"\0" + d for t, d in msgs)
        return b"OHDR" + bytes([2, 0x02]) + _u(len(body), 4) + body + b"\0" * 4

    def finish(self, links):
        lmsgs = [(0x06, bytes([1, 0, len(n)]) + n.encode() + _u(a, 8)) for n, a in links]
        root = self.alloc(self.ohdr(lmsgs))
        sb = b"\x89HDF\r\n\x1a\n" + bytes([2, 8, 8, 0]) + _u(0, 8) + _u(2**64 - 1, 8) + _u(len(self.buf), 8) + \
            _u(root, 8) + b"\0" * 4
        self.buf[:48] = sb
        return bytes(self.buf)


def _shuffle(raw: bytes, es: int) -> bytes:
    a = np.frombuffer(raw, np.uint8).reshape(-1, es)
    return a.T.tobytes()


def _filters2(es, level=4):
    # version 2: shuffle (id 2) then deflate (id 1); no names for ids < 256
    return bytes([2, 2]) + _u(2, 2) + _u(0, 2) + _u(1, 2) + _u(es, 4) + _u(1, 2) + _u(0, 2) + _u(1, 2) + _u(level, 4)


def _chunks_rowmajor(a, cd):
    grid = [-(-n // c) for n, c in zip(a.shape, cd)]
    for idx in np.ndindex(*grid):
        sl = tuple(slice(i * c, min((i + 1) * c, n)) for i, c, n in zip(idx, cd, a.shape))
        blk = np.zeros(cd, a.dtype)
        blk[tuple(slice(0, s.stop - s.start) for s in sl)] = a[sl]
        yield blk.tobytes()


def _v4_layout(index_type, cd, es, addr, extra=b"", flags=0):
    nd = len(cd) + 1
    return bytes([4, 2, flags, nd, 4]) + b"".join(_u(c, 4) for c in cd) + _u(es, 4) + bytes([index_type]) + \
        extra + _u(addr, 8)


def test_newer_structures_bit_exact(tmp_path):
    rng = np.random.default_rng(21)
    f = _V2File()
    links = []
    cls_attr = (0x0C, _attr3("MATLAB_class", b"single"))

    # fixed-array index, filtered (shuffle + deflate), edge chunks, complex compound v3
    fa = (rng.standard_normal((7, 10)) + 1j * rng.standard_normal((7, 10))).astype(np.complex64)
    cd = (3, 4)
    entries = []
    for raw in _chunks_rowmajor(fa, cd):
        z = zlib.compress(_shuffle(raw, 8), 4)
        entries.append((f.alloc(z), len(z)))
    dblk_addr = len(f.buf)
    fadb = b"FADB" + bytes([0, 1]) + _u(0, 8) + b"".join(_u(a, 8) + _u(n, 4) + _u(0, 4) for a, n in entries) + \
        b"\0" * 4
    dblk = f.alloc(fadb)
    assert dblk == dblk_addr
    fahd = b"FAHD" + bytes([0, 1, 16, 10]) + _u(len(entries), 8) + _u(dblk, 8) + b"\0" * 4
    hdr = f.alloc(fahd)
    fadb_fixed = bytearray(fadb)
    fadb_fixed[6:14] = _u(hdr, 8)
    f.buf[dblk:dblk + len(fadb)] = fadb_fixed
    oh = f.alloc(f.ohdr([(0x01, _space2(fa.shape)), (0x03, _dt_complex3(8)),
                         (0x08, _v4_layout(3, cd, 8, hdr, extra=bytes([10]))), (0x0B, _filters2(8)), cls_attr]))
    links.append(("fixed", oh))

    # implicit index, unfiltered
    im = rng.standard_normal((5, 6)).astype(np.float32)
    data = b"".join(_chunks_rowmajor(im, (2, 6)))
    a = f.alloc(data)
    oh = f.alloc(f.ohdr([(0x01, _space2(im.shape)), (0x03, _dt_float(4)), (0x08, _v4_layout(2, (2, 6), 4, a)),
                         cls_attr]))
    links.append(("implicit", oh))

    # single-chunk index, filtered
    sc = rng.standard_normal((4, 9))
    z = zlib.compress(_shuffle(sc.tobytes(), 8), 6)
    a = f.alloc(z)
    oh = f.alloc(f.ohdr([(0x01, _space2(sc.shape)), (0x03, _dt_float(8)),
                         (0x08, _v4_layout(1, sc.shape, 8, a, extra=_u(len(z), 8) + _u(0, 4), flags=2)),
                         (0x0B, _filters2(8, 6)), (0x0C, _attr3("MATLAB_class", b"double"))]))
    links.append(("single", oh))

    # compact layout (version 3)
    cp = np.arange(6, dtype=np.float64).reshape(2, 3)
    oh = f.alloc(f.ohdr([(0x01, _space2(cp.shape)), (0x03, _dt_float(8)),
                         (0x08, bytes([3, 0]) + _u(cp.nbytes, 2) + cp.tobytes())]))
    links.append(("compact", oh))

    p = tmp_path / "v2.h5"
    p.write_bytes(f.finish(links))
    with matio.H5File(str(p)) as h:
        assert sorted(h.names()) == ["compact", "fixed", "implicit", "single"]
        assert h.userblock == 0
        assert np.array_equal(h.read_raw("/fixed"), fa) and h.info("/fixed").mclass == "single"
        assert h.info("/fixed").chunk[0] == 3 and h.info("/fixed").n_filters == 2
        assert np.array_equal(h.read_raw("/implicit"), im)
        assert np.array_equal(h.read_raw("/single"), sc) and h.info("/single").mclass == "double"
        assert np.array_equal(h.read_raw("/compact"), cp) and h.info("/compact").layout == 0


def _link(name, addr):
    return bytes([1, 0, len(name)]) + name.encode() + _u(addr, 8)


def _dense_group(f, links, indirect: bool, two_level: bool):
    """A new-style group whose links live in a fractal heap (width 4, blocks of
    512 bytes up to 64 KiB, 32-bit heap offsets, 7-byte heap IDs) indexed by a
    version-2 B-tree of link-name records; returns its object-header address."""
    start, width, hdr_len = 512, 4, 4 + 1 + 8 + 4
    objs = [_link(n, a) for n, a in links]
    blocks = []                       # (heap offset of block, [(heap offset of object, bytes)])
    if not indirect:
        blocks.append((0, []))
        off = hdr_len
        for o in objs:
            blocks[0][1].append((off, o))
            off += len(o)
        assert off <= start
    else:
        # two rows of four 512-byte direct blocks; objects spread over blocks 0, 3 and 6
        per = -(-len(objs) // 3)
        for j, b in enumerate((0, 3, 6)):
            boff = b * start
            off = boff + hdr_len
            part = []
            for o in objs[j * per:(j + 1) * per]:
                part.append((off, o))
                off += len(o)
            assert off <= boff + start
            blocks.append((boff, part))
    heap_hdr_addr = len(f.buf)        # the header is written last; its address is fixed here
    f.alloc(bytes(200))
    block_addr = {}
    for boff, part in blocks:
        img = bytearray(start)
        img[:hdr_len] = b"FHDB" + bytes([0]) + _u(heap_hdr_addr, 8) + _u(boff, 4)
        for off, o in part:
            img[off - boff:off - boff + len(o)] = o
        block_addr[boff] = f.alloc(bytes(img))
    if indirect:
        entries = b"".join(_u(block_addr.get(i * start, 2**64 - 1), 8) for i in range(2 * width))
        root = f.alloc(b"FHIB" + bytes([0]) + _u(heap_hdr_addr, 8) + _u(0, 4) + entries + b"\0" * 4)
        rows = 2
    else:
        root, rows = block_addr[0], 0
    frhp = (b"FRHP" + bytes([0]) + _u(7, 2) + _u(0, 2) + bytes([0]) + _u(4096, 4) + _u(0, 8) + _u(2**64 - 1, 8) +
            _u(0, 8) + _u(2**64 - 1, 8) + b"".join(_u(0, 8) for _ in range(8)) + _u(width, 2) + _u(start, 8) +
            _u(65536, 8) + _u(32, 2) + _u(0, 2) + _u(root, 8) + _u(rows, 2) + b"\0" * 4)
    f.buf[heap_hdr_addr:heap_hdr_addr + len(frhp)] = frhp
    recs = [_u(zlib.crc32(n.encode()), 4) + bytes([0]) + _u(off, 4) + _u(len(o), 2)
            for (n, _), (off, o) in zip(links, [x for _, part in blocks for x in part])]
    node = 512
    if not two_level:
        leaf = f.alloc(b"BTLF" + bytes([0, 5]) + b"".join(recs) + b"\0" * 4)
        bt_root, nroot, depth = leaf, len(recs), 0
    else:
        # internal root with one record between two leaves
        half = len(recs) // 2
        l0 = f.alloc(b"BTLF" + bytes([0, 5]) + b"".join(recs[:half]) + b"\0" * 4)
        l1 = f.alloc(b"BTLF" + bytes([0, 5]) + b"".join(recs[half + 1:]) + b"\0" * 4)
        nb = ((node - 10) // 11).bit_length() - 1
        nb = nb // 8 + 1
        bt_root = f.alloc(b"BTIN" + bytes([0, 5]) + recs[half] + _u(l0, 8) + _u(half, nb) + _u(l1, 8) +
                          _u(len(recs) - half - 1, nb) + b"\0" * 4)
        nroot, depth = 1, 1
    bthd = f.alloc(b"BTHD" + bytes([0, 5]) + _u(node, 4) + _u(11, 2) + _u(depth, 2) + bytes([100, 40]) +
                   _u(bt_root, 8) + _u(nroot, 2) + _u(len(recs), 8) + b"\0" * 4)
    linfo = bytes([0, 0]) + _u(heap_hdr_addr, 8) + _u(bthd, 8)
    ginfo = bytes([0, 0])
    return f.alloc(f.ohdr([(0x02, linfo), (0x0A, ginfo)]))


@pytest.mark.parametrize("indirect,two_level", [(False, False), (True, False), (True, True)])
def test_dense_link_storage(tmp_path, indirect, two_level):
    rng = np.random.default_rng(31)
    f = _V2File()
    arrays, links = {}, []
    for i in range(20 if not indirect else 45):
        a = rng.standard_normal((3, i + 1))
        addr = f.alloc(a.tobytes())
        oh = f.alloc(f.ohdr([(0x01, _space2(a.shape)), (0x03, _dt_float(8)),
                             (0x08, bytes([3, 1]) + _u(addr, 8) + _u(a.nbytes, 8))]))
        arrays[f"var{i:02d}"] = a
        links.append((f"var{i:02d}", oh))
    g = _dense_group(f, links, indirect, two_level)
    p = tmp_path / "dense.h5"
    p.write_bytes(f.finish([("grp", g)]))
    with matio.H5File(str(p)) as h:
        assert h.names() == ["grp"]
        assert sorted(h.names("/grp")) == sorted(arrays)
        for k, v in arrays.items():
            assert np.array_equal(h.read_raw(f"/grp/{k}"), v), k
        assert h.info("/grp").dtype == matio.GROUP


# ───────────────────────── failures are statuses ─────────────────────────

def test_errors_are_reported(tmp_path):
    with pytest.raises(matio.MatIOError) as e:
        matio.H5File(str(tmp_path / "missing.mat"))
    assert e.value.code == matio.ERR_IO
    junk = tmp_path / "junk.mat"
    junk.write_bytes(b"MATLAB 5.0 MAT-file" + bytes(3000))
    with pytest.raises(matio.MatIOError) as e:
        matio.H5File(str(junk))
    assert e.value.code == matio.ERR_FORMAT

    p = str(tmp_path / "ok.mat")
    x = np.arange(24, dtype=np.float32).reshape(4, 6)
    matio.matwrite(p, {"x": x}, compress=True, chunk_bytes=32)
    with pytest.raises(matio.MatIOError) as e:
        matio.h5read(p, "nope")
    assert e.value.code == matio.ERR_NOTFOUND
    with matio.H5File(p) as f:
        wrong = np.empty(5, np.float32)
        rc = matio.lib.mslrio_read_at(f._h, f.lookup("/x"), wrong.ctypes.data, wrong.nbytes, 1)
        assert rc == matio.ERR_ARG

    # every truncation of a valid file fails cleanly (status, not a crash) or reads correctly
    blob = open(p, "rb").read()
    for cut in range(520, len(blob), max(1, (len(blob) - 520) // 60)):
        t = tmp_path / "cut.mat"
        t.write_bytes(blob[:cut])
        try:
            got = matio.h5read(str(t), "x")
            assert np.array_equal(got, x)
        except matio.MatIOError as err:
            assert err.code in (matio.ERR_FORMAT, matio.ERR_NOTFOUND, matio.ERR_UNSUPPORTED)

    with pytest.raises(matio.MatIOError):
        matio.matwrite(str(tmp_path / "bad.mat"), {"s": {"a": 1}})
    assert not os.path.exists(tmp_path / "bad.mat")          # a failed write leaves no partial file
    with pytest.raises(matio.MatIOError):
        with matio.MatWriter(str(tmp_path / "dup.mat")) as w:
            w.write("a", 1.0)
            w.write("a", 2.0)


_FUZZ = r"""
import os, resource, sys
import numpy as np
sys.path.insert(0, os.environ["REPO"])
resource.setrlimit(resource.RLIMIT_AS, (6 << 30, 6 << 30))
from mslr_recon_b200 import matio
src, dst = sys.argv[1], sys.argv[2]
blob = bytearray(open(src, "rb").read())
rng = np.random.default_rng(int(sys.argv[3]))
n_ok = n_err = 0
for trial in range(150):
    b = bytearray(blob)
    for _ in range(int(rng.integers(1, 4))):
        i = int(rng.integers(512, len(b)))
        b[i] = int(rng.integers(0, 256))
    open(dst, "wb").write(b)
    try:
        matio.matread(dst, nthreads=2)
        n_ok += 1
    except Exception:
        n_err += 1
print(n_ok, n_err)
"""


def test_damaged_files_never_crash(tmp_path):
    """Random byte changes in a valid file (outside the MATLAB header) give a
    result or an exception, never a crash; run in a child process whose
    address space is capped, so that an absurd size read from the damage
    fails as an allocation error instead of exhausting memory."""
    import subprocess
    import sys
    rng = np.random.default_rng(17)
    d = {"x": (rng.standard_normal((4, 6, 5)) + 1j * rng.standard_normal((4, 6, 5))).astype(np.complex64),
         "c": [np.arange(3.0), "abc"], "m": rng.random((5, 5)) > 0.5, "s": 3.5}
    src = str(tmp_path / "src.mat")
    matio.matwrite(src, d, compress=True, chunk_bytes=64)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = tmp_path / "fuzz.py"
    script.write_text(_FUZZ)
    for seed in (1, 2):
        r = subprocess.run([sys.executable, str(script), src, str(tmp_path / "dst.mat"), str(seed)],
                           capture_output=True, text=True, timeout=300, env={**os.environ, "REPO": root})
        assert r.returncode == 0, (r.returncode, r.stderr[-2000:])
        ok, err = (int(v) for v in r.stdout.split())
        assert ok + err == 150


_C_PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "mslr_io.h"
int main(int argc, char** argv) {
    float data[2 * 3 * 4 * 2];
    for (int i = 0; i < 48; ++i) data[i] = (float)i - 7.5f;
    int64_t dims[3] = {2, 3, 4};
    mslrio_writer* w = NULL;
    uint64_t a = 0;
    if (mslrio_create(argv[1], 1, &w)) return 1;
    if (mslrio_write(w, "ksp_epi_zf", MSLRIO_C64, 3, dims, data, "single", -1, 0, 6, 32, 2, &a)) return 2;
    if (mslrio_finish(w)) return 3;
    mslrio_file* f = NULL;
    if (mslrio_open(argv[1], &f)) return 4;
    uint64_t addr = 0;
    mslrio_info info;
    if (mslrio_lookup(f, "/ksp_epi_zf", &addr) || addr != a) return 5;
    if (mslrio_info_at(f, addr, &info) || info.dtype != MSLRIO_C64 || info.rank != 3 || info.layout != 2) return 6;
    if (strcmp(info.matlab_class, "single")) return 7;
    float back[48];
    if (mslrio_read_at(f, addr, back, sizeof(back), 0)) return 8;
    if (memcmp(back, data, sizeof(back))) return 9;
    if (mslrio_read_at(f, addr, back, 8, 1) != MSLRIO_ERR_ARG || !strlen(mslrio_last_error())) return 10;
    if (mslrio_lookup(f, "/nope", &addr) != MSLRIO_ERR_NOTFOUND) return 11;
    mslrio_close(f);
    printf("ok\n");
    return 0;
}
"""


def test_c_header_from_c(tmp_path):
    """include/mslr_io.h is plain C99 and the library works from a C program."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "t.c"
    src.write_text(_C_PROGRAM)
    exe = tmp_path / "t"
    libdir = os.path.dirname(matio._LIB_PATH)
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(root, "include"), str(src), "-o",
                        str(exe), "-L", libdir, "-l:libmslrio.so", "-Wl,-rpath," + libdir],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe), str(tmp_path / "c.mat")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout, r.stderr)
    b, _ = H.OracleFile(str(tmp_path / "c.mat")).read("/ksp_epi_zf")
    want = (np.arange(48, dtype=np.float32) - 7.5).view(np.complex64).reshape(2, 3, 4)
    assert np.array_equal(b, want)


def test_c_abi_exports():
    import ctypes
    lib = ctypes.CDLL(matio._LIB_PATH)
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "mslr_io.h")).read()
    import re
    names = set(re.findall(r"\b(mslrio_[a-z_]+)\s*\(", hdr))
    assert len(names) == 13
    for n in names:
        assert hasattr(lib, n), n
