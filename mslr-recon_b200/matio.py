"""MAT v7.3 / HDF5 files for run_recon: h5read, matread and matwrite.

The reference reads its inputs and writes its results through Julia
packages on libhdf5 (scripts/reconstruct.jl:88 ``matread(fn_smaps)["smaps"]``,
:95 ``h5read(fn_ksp, "ksp_epi_zf")``, :242-260 ``matwrite(fn_out, Dict(...);
compress=true)``).  Here the same calls sit on ``libmslrio.so``
(``include/mslr_io.h``), a host-threaded reader and writer of the HDF5
structures those files use.

Array convention: HDF5 stores a Julia / MATLAB array of size (d1, ..., dn)
with dims (dn, ..., d1) and the same bytes, so the numpy arrays here are
C-ordered with the dims reversed — exactly the layouts the rest of this
package takes (k-space (Nt, Nc, Nz, Ny, Nx), coil maps (Nc, Nz, Ny, Nx),
X (Ns, Nt, Nz, Ny, Nx)).  A 1-D numpy array is written as a MATLAB column
vector (HDF5 dims (1, n)); a 1×1 MATLAB array reads back as a Python scalar,
as MAT.jl returns it.
"""
from __future__ import annotations

import ctypes as C
import os
import string

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmslrio.so")

OK, ERR_ARG, ERR_IO, ERR_FORMAT, ERR_UNSUPPORTED, ERR_NOTFOUND = 0, 1, 2, 3, 4, 5
I8, U8, I16, U16, I32, U32, I64, U64, F32, F64, C64, C128, REF, STR = range(1, 15)
GROUP = 100
MAX_RANK = 32

_NP = {I8: np.int8, U8: np.uint8, I16: np.int16, U16: np.uint16, I32: np.int32, U32: np.uint32,
       I64: np.int64, U64: np.uint64, F32: np.float32, F64: np.float64, C64: np.complex64,
       C128: np.complex128, REF: np.uint64}
_CODE = {np.dtype(v): k for k, v in _NP.items() if k != REF}
_MCLASS = {I8: "int8", U8: "uint8", I16: "int16", U16: "uint16", I32: "int32", U32: "uint32",
           I64: "int64", U64: "uint64", F32: "single", F64: "double", C64: "single", C128: "double"}


class MatIOError(RuntimeError):
    """A failed libmslrio call; ``code`` is the MSLRIO_ERR_* status."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class Info(C.Structure):
    _fields_ = [("addr", C.c_uint64), ("dtype", C.c_int32), ("elem_size", C.c_int32),
                ("rank", C.c_int32), ("layout", C.c_int32), ("dims", C.c_int64 * MAX_RANK),
                ("chunk", C.c_int64 * MAX_RANK), ("n_filters", C.c_int32),
                ("matlab_int_decode", C.c_int32), ("matlab_empty", C.c_int32),
                ("matlab_class", C.c_char * 32)]

    @property
    def shape(self):
        return tuple(int(self.dims[d]) for d in range(self.rank))

    @property
    def mclass(self) -> str:
        return self.matlab_class.decode()


def _load():
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} is missing: run mslr-recon_b200/build_lib.py")
    lib = C.CDLL(_LIB_PATH)
    P, I32_, I64_, SZ, U64P = C.c_void_p, C.c_int32, C.c_int64, C.c_size_t, C.POINTER(C.c_uint64)
    lib.mslrio_open.argtypes = [C.c_char_p, C.POINTER(P)]
    lib.mslrio_close.argtypes = [P]
    lib.mslrio_userblock.argtypes = [P, U64P]
    lib.mslrio_group_count.argtypes = [P, C.c_char_p, C.POINTER(I32_)]
    lib.mslrio_group_name.argtypes = [P, C.c_char_p, I32_, C.c_char_p, SZ]
    lib.mslrio_lookup.argtypes = [P, C.c_char_p, U64P]
    lib.mslrio_info_at.argtypes = [P, C.c_uint64, C.POINTER(Info)]
    lib.mslrio_read_at.argtypes = [P, C.c_uint64, P, SZ, I32_]
    lib.mslrio_create.argtypes = [C.c_char_p, I32_, C.POINTER(P)]
    lib.mslrio_write.argtypes = [P, C.c_char_p, I32_, I32_, C.POINTER(I64_), P, C.c_char_p, I32_, I32_,
                                 I32_, I64_, I32_, U64P]
    lib.mslrio_finish.argtypes = [P]
    lib.mslrio_abort.argtypes = [P]
    lib.mslrio_last_error.restype = C.c_char_p
    return lib


lib = _load()


def _chk(rc: int):
    if rc != OK:
        raise MatIOError(rc, lib.mslrio_last_error().decode(errors="replace"))


class H5File:
    """A read-only HDF5 / MAT v7.3 file (memory-mapped by libmslrio)."""

    def __init__(self, path: str, nthreads: int = 0):
        self._h = C.c_void_p()
        _chk(lib.mslrio_open(os.fsencode(path), C.byref(self._h)))
        self.nthreads = int(nthreads)

    def close(self):
        if self._h:
            lib.mslrio_close(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()

    @property
    def userblock(self) -> int:
        v = C.c_uint64()
        _chk(lib.mslrio_userblock(self._h, C.byref(v)))
        return int(v.value)

    def names(self, group: str = "/"):
        n = C.c_int32()
        _chk(lib.mslrio_group_count(self._h, group.encode(), C.byref(n)))
        buf = C.create_string_buffer(4096)
        out = []
        for i in range(n.value):
            _chk(lib.mslrio_group_name(self._h, group.encode(), i, buf, len(buf)))
            out.append(buf.value.decode())
        return out

    def lookup(self, path: str) -> int:
        a = C.c_uint64()
        _chk(lib.mslrio_lookup(self._h, path.encode(), C.byref(a)))
        return int(a.value)

    def info(self, path_or_addr) -> Info:
        addr = self.lookup(path_or_addr) if isinstance(path_or_addr, str) else int(path_or_addr)
        inf = Info()
        _chk(lib.mslrio_info_at(self._h, addr, C.byref(inf)))
        return inf

    def read_raw(self, path_or_addr) -> np.ndarray:
        """The dataset's elements as stored: a C-order array with the HDF5
        dims (complex pairs as complex64/128, references as uint64
        addresses, strings as an 'S<n>' array)."""
        inf = self.info(path_or_addr)
        if inf.dtype == GROUP:
            raise MatIOError(ERR_ARG, "object is a group")
        dt = np.dtype(f"S{inf.elem_size}") if inf.dtype == STR else np.dtype(_NP[inf.dtype])
        out = np.empty(inf.shape, dtype=dt)
        _chk(lib.mslrio_read_at(self._h, inf.addr, out.ctypes.data_as(C.c_void_p), out.nbytes, self.nthreads))
        return out

    def read_matlab(self, path_or_addr):
        """A MATLAB variable decoded as matread does: numeric arrays, logical
        → bool, char → str, cell → list, struct → dict, 1×1 → scalar."""
        inf = self.info(path_or_addr)
        cls = inf.mclass
        if inf.dtype == GROUP:
            if cls and cls != "struct":
                raise MatIOError(ERR_UNSUPPORTED, f"MATLAB class {cls!r} stored as a group")
            base = path_or_addr if isinstance(path_or_addr, str) else None
            if base is None:
                raise MatIOError(ERR_UNSUPPORTED, "structs inside cells are not supported")
            return {n: self.read_matlab(base.rstrip("/") + "/" + n) for n in self.names(base)}
        if inf.matlab_empty:
            mdims = tuple(int(v) for v in self.read_raw(inf.addr).ravel())
            dt = {"char": np.uint16, "logical": np.bool_, "cell": object}.get(cls, np.float64)
            if cls in _MCLASS.values() and cls not in ("single", "double"):
                dt = np.dtype(cls)
            elif cls == "single":
                dt = np.float32
            return "" if cls == "char" else np.zeros(tuple(reversed(mdims)), dtype=dt)
        a = self.read_raw(inf.addr)
        if cls == "cell":
            return [self.read_matlab(int(r)) for r in a.ravel()]
        if cls == "char":       # MATLAB char: UTF-16 code units, column-major
            return np.ascontiguousarray(a.T).astype("<u2").tobytes().decode("utf-16-le", errors="replace")
        if cls == "logical":
            a = a.astype(np.bool_)
        if a.size == 1 and a.ndim == 2:
            return a.reshape(()).item()
        return a


def h5read(path: str, name: str, nthreads: int = 0) -> np.ndarray:
    """HDF5.jl's ``h5read(path, name)``: the whole dataset, C order, HDF5
    dims (scripts/reconstruct.jl:95 reads ``ksp_epi_zf`` this way; its
    compound {real, imag} elements come back as complex64)."""
    with H5File(path, nthreads) as f:
        return f.read_raw(name if name.startswith("/") else "/" + name)


def is_hdf5(path: str) -> bool:
    with open(path, "rb") as fh:
        head = fh.read(2048 + 8)
    sig = b"\x89HDF\r\n\x1a\n"
    return any(head[o:o + 8] == sig for o in (0, 512, 1024, 2048))


def matread(path: str, nthreads: int = 0) -> dict:
    """MAT.jl's ``matread(path)``: every top-level variable, decoded.  v7.3
    (HDF5) files are read by libmslrio; v4-v7 files by scipy.io.loadmat,
    with their arrays in the same reversed-dims convention."""
    if is_hdf5(path):
        with H5File(path, nthreads) as f:
            return {n: f.read_matlab("/" + n) for n in f.names("/") if not n.startswith("#")}
    from scipy.io import loadmat
    out = {}
    for k, v in loadmat(path, mat_dtype=False, squeeze_me=False, chars_as_strings=True).items():
        if k.startswith("__"):
            continue
        if isinstance(v, np.ndarray) and v.dtype.kind in "biufc":
            v = v.T
            if v.size == 1 and v.ndim == 2:
                v = v.reshape(()).item()
        out[k] = v
    return out


def _refs_name(i: int) -> str:
    letters = string.ascii_lowercase
    s = ""
    i += 1
    while i > 0:
        i, r = divmod(i - 1, 26)
        s = letters[r] + s
    return s


class MatWriter:
    """Writes a MAT v7.3 file variable by variable (see :func:`matwrite`)."""

    def __init__(self, path: str, compress: bool = False, level: int = 3, nthreads: int = 0,
                 chunk_bytes: int = 4 << 20):
        self._h = C.c_void_p()
        _chk(lib.mslrio_create(os.fsencode(path), 1, C.byref(self._h)))
        self.level = int(level) if compress else 0
        self.nthreads = int(nthreads)
        self.chunk_bytes = int(chunk_bytes)
        self._nrefs = 0

    def _put(self, name: str, a: np.ndarray, code: int, mclass: str, int_decode: int = -1,
             empty: int = 0) -> int:
        a = np.ascontiguousarray(a)
        dims = (C.c_int64 * max(1, a.ndim))(*a.shape)
        addr = C.c_uint64()
        _chk(lib.mslrio_write(self._h, name.encode(), code, a.ndim, dims, a.ctypes.data_as(C.c_void_p),
                              mclass.encode(), int_decode, empty, self.level if a.size else 0,
                              self.chunk_bytes, self.nthreads, C.byref(addr)))
        return int(addr.value)

    def write(self, name: str, v) -> int:
        """Write one variable; returns its object address."""
        if isinstance(v, dict):
            raise MatIOError(ERR_UNSUPPORTED, "struct values are not supported by matwrite here")
        if isinstance(v, str):
            if not v:
                return self._put(name, np.array([0, 0], dtype=np.uint64), U64, "char", 2, 1)
            codes = np.frombuffer(v.encode("utf-16-le"), dtype="<u2")
            return self._put(name, codes.reshape(codes.size, 1), U16, "char", 2)
        if isinstance(v, (list, tuple)):
            refs = []
            for item in v:
                refs.append(self.write(f"#refs#/{_refs_name(self._nrefs)}", item))
                self._nrefs += 1
            arr = np.array(refs, dtype=np.uint64).reshape(1, len(refs))
            if not refs:
                return self._put(name, np.array([0, 0], dtype=np.uint64), U64, "cell", -1, 1)
            return self._put(name, arr, REF, "cell")
        a = np.asarray(v)
        if a.ndim == 0:
            a = a.reshape(1, 1)
        elif a.ndim == 1:
            a = a.reshape(1, a.shape[0])        # MATLAB column vector (n × 1)
        if a.dtype == np.bool_:
            if a.size == 0:
                return self._put(name, np.array(a.shape[::-1], dtype=np.uint64), U64, "logical", 1, 1)
            return self._put(name, a.astype(np.uint8), U8, "logical", 1)
        if a.dtype not in _CODE:
            raise MatIOError(ERR_UNSUPPORTED, f"cannot write {name!r} of dtype {a.dtype}")
        code = _CODE[a.dtype]
        if a.size == 0:
            return self._put(name, np.array(a.shape[::-1], dtype=np.uint64), U64, _MCLASS[code], -1, 1)
        return self._put(name, a, code, _MCLASS[code])

    def close(self):
        if self._h:
            h, self._h = self._h, C.c_void_p()
            _chk(lib.mslrio_finish(h))

    def abort(self):
        if self._h:
            h, self._h = self._h, C.c_void_p()
            lib.mslrio_abort(h)

    def __enter__(self):
        return self

    def __exit__(self, exc_type, *exc):
        if exc_type is None:
            self.close()
        else:
            self.abort()


def matwrite(path: str, d: dict, compress: bool = False, nthreads: int = 0, level: int = 3,
             chunk_bytes: int = 4 << 20):
    """MAT.jl's ``matwrite(path, Dict(...); compress)`` (scripts/reconstruct.jl:
    242-260): a MAT v7.3 file with one variable per key.  Values: numpy
    arrays (any int / float / complex / bool dtype), Python scalars, str,
    and lists (cell arrays, stored under ``#refs#`` as MATLAB does).
    ``compress`` stores arrays in deflate-compressed chunks of about
    chunk_bytes, compressed on ``nthreads`` host threads."""
    with MatWriter(path, compress, level, nthreads, chunk_bytes) as w:
        for k, v in d.items():
            w.write(k, v)
