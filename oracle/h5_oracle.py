"""Independent pure-Python HDF5 reader — test infrastructure only.

This is the checker for ``libmslrio.so`` (the product's MAT v7.3 reader and
writer).  It restates, separately from the C++ code, the part of the
published HDF5 file-format specification that MAT v7.3 files use, so that
files written by the library are decoded by a second implementation:

- superblock versions 0 and 1 (root group symbol-table entry);
- version-1 object headers with continuation messages;
- symbol-table groups (version-1 group B-tree, symbol-table nodes, local
  heap names);
- dataspace message version 1 and 2; datatypes: fixed point, IEEE float,
  compound (complex pairs), string, object reference;
- data layout messages version 1-3: compact, contiguous, chunked with a
  version-1 chunk B-tree; deflate and shuffle filters with the per-chunk
  filter mask;
- attributes (version 1) for MATLAB_class / MATLAB_int_decode / MATLAB_empty.

The reference itself reads these files through HDF5.jl and MAT.jl on
libhdf5 (scripts/reconstruct.jl:88,95; its output at :242-260).  Neither
Julia nor libhdf5 exists in this image, so the pin for both this reader and
the library is a MATLAB-written v7.3 file shipped with scipy's test data
(``testhdf5_7.4_GLNX86.mat``: variable ``testdouble`` = 0:pi/4:2*pi), plus
agreement between the two implementations on every file the library writes.
Only ``tests/`` imports this module.
"""
from __future__ import annotations

import zlib

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5OracleError(Exception):
    pass


def _u(b: bytes, o: int, n: int) -> int:
    return int.from_bytes(b[o:o + n], "little")


class OracleFile:
    def __init__(self, path: str):
        with open(path, "rb") as fh:
            self.b = fh.read()
        b = self.b
        self.sb = None
        o = 0
        while o + 8 <= len(b):
            if b[o:o + 8] == SIG:
                self.sb = o
                break
            o = 512 if o == 0 else o * 2
        if self.sb is None:
            raise H5OracleError("no HDF5 signature")
        ver = b[self.sb + 8]
        if ver not in (0, 1):
            raise H5OracleError(f"superblock version {ver} outside the oracle's subset")
        self.so, self.sl = b[self.sb + 13], b[self.sb + 14]
        self.leaf_k = _u(b, self.sb + 16, 2)
        self.internal_k = _u(b, self.sb + 18, 2)
        p = self.sb + 24 + (4 if ver == 1 else 0)
        self.base_field = _u(b, p, self.so)
        self.eof_field = _u(b, p + 2 * self.so, self.so)
        root_entry = p + 4 * self.so
        self.root = _u(b, root_entry + self.so, self.so)

    # absolute file offset of a file address
    def abs(self, addr: int) -> int:
        a = self.sb + addr
        if addr == UNDEF or a >= len(self.b):
            raise H5OracleError("address outside the file")
        return a

    def messages(self, addr: int):
        b = self.b
        a = self.abs(addr)
        if b[a] != 1:
            raise H5OracleError("object header version outside the oracle's subset")
        nmsgs = _u(b, a + 2, 2)
        hsize = _u(b, a + 8, 4)
        blocks = [(a + 16, a + 16 + hsize)]
        out = []
        seen = 0
        while blocks:
            lo, hi = blocks.pop(0)
            p = lo
            while p + 8 <= hi:
                mtype, msize, mflags = _u(b, p, 2), _u(b, p + 2, 2), b[p + 4]
                data = b[p + 8:p + 8 + msize]
                seen += 1
                if mtype == 0x10:
                    ca, cl = _u(data, 0, self.so), _u(data, self.so, self.sl)
                    blocks.append((self.abs(ca), self.abs(ca) + cl))
                else:
                    out.append((mtype, mflags, data))
                p += 8 + msize
        # the prefix's message count covers every message, continuations included
        if seen != nmsgs:
            raise H5OracleError(f"object header declares {nmsgs} messages and holds {seen}")
        return out

    def members(self, addr: int):
        msgs = self.messages(addr)
        stab = [d for t, _, d in msgs if t == 0x11]
        if not stab:
            raise H5OracleError("not a symbol-table group")
        bt, heap = _u(stab[0], 0, self.so), _u(stab[0], self.so, self.so)
        b = self.b
        h = self.abs(heap)
        if b[h:h + 4] != b"HEAP":
            raise H5OracleError("bad local heap")
        dseg = self.abs(_u(b, h + 8 + 2 * self.sl, self.so))
        out = []

        def walk(node):
            n = self.abs(node)
            if b[n:n + 4] != b"TREE" or b[n + 4] != 0:
                raise H5OracleError("bad group B-tree node")
            level, used = b[n + 5], _u(b, n + 6, 2)
            p = n + 8 + 2 * self.so
            for _ in range(used):
                p += self.sl
                child = _u(b, p, self.so)
                p += self.so
                if level > 0:
                    walk(child)
                    continue
                s = self.abs(child)
                if b[s:s + 4] != b"SNOD":
                    raise H5OracleError("bad symbol-table node")
                for k in range(_u(b, s + 6, 2)):
                    e = s + 8 + k * (2 * self.so + 24)
                    noff, oh = _u(b, e, self.so), _u(b, e + self.so, self.so)
                    name = b[dseg + noff:b.index(b"\0", dseg + noff)].decode()
                    out.append((name, oh))

        walk(bt)
        return out

    def lookup(self, path: str) -> int:
        cur = self.root
        for part in [p for p in path.split("/") if p]:
            d = dict(self.members(cur))
            if part not in d:
                raise KeyError(path)
            cur = d[part]
        return cur

    # ── datatypes ──
    def dtype(self, d: bytes, o: int = 0):
        """Returns (numpy dtype or tag, size, bytes consumed)."""
        cls, ver = d[o] & 15, d[o] >> 4
        bf = _u(d, o + 1, 3)
        size = _u(d, o + 4, 4)
        p = o + 8
        if cls == 0:
            if bf & 1:
                raise H5OracleError("big-endian integers")
            kind = "i" if bf & 8 else "u"
            return np.dtype(f"<{kind}{size}"), size, 8 + 4
        if cls == 1:
            return np.dtype(f"<f{size}"), size, 8 + 12
        if cls == 3:
            return np.dtype(f"S{size}"), size, 8
        if cls == 7:
            return np.dtype("<u8"), size, 8
        if cls == 6:
            names, offs, types = [], [], []
            for _ in range(bf & 0xFFFF):
                end = d.index(b"\0", p)
                names.append(d[p:end].decode())
                p += ((end - p + 1 + 7) // 8) * 8 if ver < 3 else end - p + 1
                offs.append(_u(d, p, 4))
                p += 4 + (28 if ver == 1 else 0)
                t, _, used = self.dtype(d, p)
                types.append(t)
                p += used
            if len(names) == 2 and types[0] == types[1] and types[0].kind == "f" and offs == [0, types[0].itemsize]:
                return np.dtype(f"<c{2 * types[0].itemsize}"), size, p - o
            raise H5OracleError("compound other than a complex pair")
        raise H5OracleError(f"datatype class {cls}")

    @staticmethod
    def space(d: bytes, sl: int):
        ver, rank = d[0], d[1]
        p = 8 if ver == 1 else 4
        return tuple(_u(d, p + i * sl, sl) for i in range(rank))

    def attributes(self, msgs):
        out = {}
        for t, _, d in msgs:
            if t != 0x0C or d[0] != 1:
                continue
            nl, tl, sl_ = _u(d, 2, 2), _u(d, 4, 2), _u(d, 6, 2)
            p = 8
            name = d[p:p + nl].rstrip(b"\0").decode()
            p += (nl + 7) // 8 * 8
            dt, size, _ = self.dtype(d, p)
            p += (tl + 7) // 8 * 8
            p += (sl_ + 7) // 8 * 8
            raw = d[p:p + size]
            out[name] = raw.rstrip(b"\0").decode() if dt.kind == "S" else int.from_bytes(raw, "little")
        return out

    def read(self, path_or_addr):
        """(array with the HDF5 dims, attributes) of one dataset."""
        addr = self.lookup(path_or_addr) if isinstance(path_or_addr, str) else path_or_addr
        msgs = self.messages(addr)
        by = {}
        for t, _, d in msgs:
            by.setdefault(t, d)
        dims = self.space(by[0x01], self.sl)
        dt, esize, _ = self.dtype(by[0x03])
        lay = by[0x08]
        filters = []
        if 0x0B in by:
            f = by[0x0B]
            p = 8 if f[0] == 1 else 2
            for _ in range(f[1]):
                fid, nl, nv = _u(f, p, 2), _u(f, p + 2, 2), _u(f, p + 6, 2)
                p += 8 + ((nl + 7) // 8 * 8 if f[0] == 1 else nl)
                cd = [_u(f, p + 4 * i, 4) for i in range(nv)]
                p += 4 * nv + (4 if f[0] == 1 and nv % 2 else 0)
                filters.append((fid, cd))
        n = int(np.prod(dims)) if dims else 1
        nbytes = n * esize
        ver = lay[0]
        if ver == 3:
            cls = lay[1]
            if cls == 0:
                raw = lay[4:4 + _u(lay, 2, 2)]
            elif cls == 1:
                a = _u(lay, 2, self.so)
                raw = bytes(nbytes) if a == UNDEF else self.b[self.abs(a):self.abs(a) + nbytes]
            else:
                nd = lay[2]
                bt = _u(lay, 3, self.so)
                cdims = [_u(lay, 3 + self.so + 4 * i, 4) for i in range(nd)]
                return self._chunked(dims, dt, esize, cdims[:-1], bt, filters), self.attributes(msgs)
        elif ver in (1, 2):
            nd, cls = lay[1], lay[2]
            if cls == 2:
                bt = _u(lay, 8, self.so)
                cdims = [_u(lay, 8 + self.so + 4 * i, 4) for i in range(nd)]
                return self._chunked(dims, dt, esize, cdims[:-1], bt, filters), self.attributes(msgs)
            a = _u(lay, 8, self.so)
            raw = self.b[self.abs(a):self.abs(a) + nbytes]
        else:
            raise H5OracleError(f"layout version {ver}")
        arr = np.frombuffer(raw, dtype=dt, count=n).reshape(dims) if n else np.zeros(dims, dt)
        return arr.copy(), self.attributes(msgs)

    def _chunked(self, dims, dt, esize, cdims, bt, filters):
        b = self.b
        rank = len(dims)
        out = np.zeros(dims, dtype=dt)
        csize = int(np.prod(cdims)) * esize
        recs = []

        def walk(node):
            n = self.abs(node)
            if b[n:n + 4] != b"TREE" or b[n + 4] != 1:
                raise H5OracleError("bad chunk B-tree node")
            level, used = b[n + 5], _u(b, n + 6, 2)
            p = n + 8 + 2 * self.so
            for _ in range(used):
                size, mask = _u(b, p, 4), _u(b, p + 4, 4)
                offs = [_u(b, p + 8 + 8 * i, 8) for i in range(rank + 1)]
                p += 8 + 8 * (rank + 1)
                child = _u(b, p, self.so)
                p += self.so
                if level > 0:
                    walk(child)
                else:
                    recs.append((child, size, mask, offs[:rank]))

        walk(bt)
        for addr, size, mask, offs in recs:
            raw = self.b[self.abs(addr):self.abs(addr) + size]
            for i in reversed(range(len(filters))):
                if mask & (1 << i):
                    continue
                fid, cd = filters[i]
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:
                    es = cd[0] if cd else 1
                    a = np.frombuffer(raw[:len(raw) // es * es], np.uint8).reshape(es, -1).T.reshape(-1)
                    raw = a.tobytes() + raw[len(raw) // es * es:]
                else:
                    raise H5OracleError(f"filter {fid}")
            if len(raw) != csize:
                raise H5OracleError("chunk decodes to the wrong size")
            chunk = np.frombuffer(raw, dtype=dt).reshape(cdims)
            sl_out = tuple(slice(o, min(o + c, d)) for o, c, d in zip(offs, cdims, dims))
            sl_in = tuple(slice(0, s.stop - s.start) for s in sl_out)
            out[sl_out] = chunk[sl_in]
        return out


def matlab_header(path: str):
    """(text, version bytes, endian indicator) of a MAT v7.3 user block."""
    with open(path, "rb") as fh:
        ub = fh.read(128)
    return ub[:116].decode("ascii", "replace"), ub[124:126], ub[126:128]
