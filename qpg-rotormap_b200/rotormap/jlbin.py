"""The reference's index file format: a Julia `Serialization` stream of one
NamedTuple (`save` / `load`, RotorMap/common/dna.jl:23-34; the NamedTuple of
_index_data_nt, RotorMap/index/build.jl:755-772).

Parsing and writing run in the library (r2m_jlbin_*, csrc/jlser.cpp); this
module turns the fields into Python values:

  Int64 -> int, Bool -> bool, String -> str,
  Array{T,N} of a bits type -> a read-only numpy memory map of the file
      (numpy shape = the Julia dims reversed, so a column-major (rdim, N)
      matrix reads as an (N, rdim) row-major array -- each Julia column is a
      numpy row),
  Vector{String} -> StrVec (distinct strings + one index per element).

Writing takes the same values; wrap an e4m3 byte array in `E4M3` so it is
written as Matrix{Float8_E4M3FN}.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from ._lib import R2MError, R2M_EINVAL, check, lib

KIND_OTHER, KIND_INT, KIND_BOOL, KIND_STRING, KIND_ARRAY, KIND_STRVEC = 0, 1, 2, 3, 4, 5
ELTY_U8, ELTY_I32, ELTY_I64, ELTY_F16, ELTY_F32, ELTY_F64, ELTY_E4M3 = 1, 2, 3, 4, 5, 6, 7

_DTYPES = {ELTY_U8: np.uint8, ELTY_I32: np.int32, ELTY_I64: np.int64, ELTY_F16: np.float16,
           ELTY_F32: np.float32, ELTY_F64: np.float64, ELTY_E4M3: np.uint8}
_ELTYS = {np.dtype(np.uint8): ELTY_U8, np.dtype(np.int32): ELTY_I32, np.dtype(np.int64): ELTY_I64,
          np.dtype(np.float16): ELTY_F16, np.dtype(np.float32): ELTY_F32, np.dtype(np.float64): ELTY_F64}

JULIA_MAGIC = b"\x37JL"  # HEADER tag, then "JL"


class JlField(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("kind", ctypes.c_int), ("elty", ctypes.c_int),
                ("ival", ctypes.c_int64), ("str", ctypes.c_void_p), ("str_len", ctypes.c_int64),
                ("ndims", ctypes.c_int), ("dims", ctypes.c_int64 * 2), ("data", ctypes.c_void_p),
                ("offset", ctypes.c_int64), ("blob", ctypes.c_void_p), ("uniq_off", ctypes.c_void_p),
                ("nuniq", ctypes.c_int64)]


@dataclass
class StrVec:
    """A Vector{String}: element i is uniq[idx[i]]."""
    uniq: list
    idx: np.ndarray  # int32

    def __len__(self) -> int:
        return int(self.idx.size)

    def tolist(self) -> list:
        return [self.uniq[i] for i in self.idx]

    @classmethod
    def from_list(cls, items) -> "StrVec":
        ids, uniq = {}, []
        idx = np.empty(len(items), np.int32)
        for i, s in enumerate(items):
            j = ids.get(s)
            if j is None:
                j = ids[s] = len(uniq)
                uniq.append(s)
            idx[i] = j
        return cls(uniq, idx)


class E4M3:
    """An e4m3 byte array to be written as Array{Float8_E4M3FN}."""

    def __init__(self, a):
        self.a = np.ascontiguousarray(a, dtype=np.uint8)


def _strings(f: JlField) -> StrVec:
    n = int(f.dims[0])
    idx = np.ctypeslib.as_array((ctypes.c_int32 * n).from_address(f.data)).copy() if n else np.zeros(0, np.int32)
    nu = int(f.nuniq)
    offs = np.ctypeslib.as_array((ctypes.c_int64 * (nu + 1)).from_address(f.uniq_off)).copy() if nu else [0]
    blob = ctypes.string_at(f.blob, int(offs[-1])) if nu and offs[-1] else b""
    uniq = [blob[offs[i]:offs[i + 1]].decode("utf-8", "surrogateescape") for i in range(nu)]
    return StrVec(uniq, idx)


def read_bin(path, mmap: bool = True) -> tuple[dict, int]:
    """Parse an index .bin: ({field name: value}, format version byte).
    Arrays are memory maps of the file (mmap=True) or in-memory copies."""
    path = os.fspath(path)
    L = lib()
    h = ctypes.c_void_p()
    check(L.r2m_jlbin_open(path.encode(), ctypes.byref(h)))
    out = {}
    try:
        ver = int(L.r2m_jlbin_version(h))
        for i in range(int(L.r2m_jlbin_nfields(h))):
            f = JlField()
            check(L.r2m_jlbin_field(h, i, ctypes.byref(f)))
            name = f.name.decode()
            if f.kind == KIND_INT:
                v = int(f.ival)
            elif f.kind == KIND_BOOL:
                v = bool(f.ival)
            elif f.kind == KIND_STRING:
                v = ctypes.string_at(f.str, f.str_len).decode("utf-8", "surrogateescape") if f.str_len else ""
            elif f.kind == KIND_ARRAY:
                dt = _DTYPES.get(f.elty)
                if dt is None:
                    raise R2MError(R2M_EINVAL, f"field {name}: unsupported element type")
                shape = tuple(int(f.dims[d]) for d in range(f.ndims))[::-1]
                count = int(np.prod(shape)) if shape else 0
                if count == 0:
                    v = np.zeros(shape, dt)
                elif mmap:
                    v = np.memmap(path, dtype=dt, mode="r", offset=int(f.offset), shape=shape)
                else:
                    nbytes = count * np.dtype(dt).itemsize
                    v = np.frombuffer(ctypes.string_at(f.data, nbytes), dt).reshape(shape)
                if f.elty == ELTY_E4M3:
                    v = E4M3Array(v)
            elif f.kind == KIND_STRVEC:
                v = _strings(f)
            else:
                v = None
            out[name] = v
    finally:
        L.r2m_jlbin_close(h)
    return out, ver


class E4M3Array(np.ndarray):
    """A uint8 view of a Float8_E4M3FN array read from a .bin (marks the
    element type, so the loader can check it like the reference does)."""

    def __new__(cls, a):
        return np.asarray(a).view(cls)


def write_bin(path, fields) -> None:
    """Write [(name, value), ...] as one NamedTuple, in order (see module doc)."""
    path = os.fspath(path)
    n = len(fields)
    arr = (JlField * n)()
    keep = []
    for i, (name, v) in enumerate(fields):
        f = arr[i]
        bname = name.encode()
        keep.append(bname)
        f.name = bname
        if isinstance(v, (bool, np.bool_)):
            f.kind, f.ival = KIND_BOOL, int(bool(v))
        elif isinstance(v, (int, np.integer)):
            f.kind, f.ival = KIND_INT, int(v)
        elif isinstance(v, str):
            b = v.encode("utf-8", "surrogateescape")
            buf = ctypes.create_string_buffer(b, len(b))
            keep.append(buf)
            f.kind, f.str, f.str_len = KIND_STRING, ctypes.addressof(buf), len(b)
        elif isinstance(v, (E4M3, E4M3Array, np.ndarray)):
            if isinstance(v, E4M3):
                a, elty = v.a, ELTY_E4M3
            elif isinstance(v, E4M3Array):
                a, elty = np.ascontiguousarray(v.view(np.ndarray)), ELTY_E4M3
            else:
                a = np.ascontiguousarray(v)
                elty = _ELTYS.get(a.dtype)
                if elty is None:
                    raise R2MError(R2M_EINVAL, f"field {name}: unsupported dtype {a.dtype}")
            if a.ndim not in (1, 2):
                raise R2MError(R2M_EINVAL, f"field {name}: 1-D or 2-D arrays only")
            keep.append(a)
            f.kind, f.elty, f.ndims = KIND_ARRAY, elty, a.ndim
            for d, s in enumerate(a.shape[::-1]):
                f.dims[d] = s
            f.data = a.ctypes.data if a.size else None
        elif isinstance(v, (StrVec, list, tuple)):
            sv = v if isinstance(v, StrVec) else StrVec.from_list(list(v))
            enc = [s.encode("utf-8", "surrogateescape") for s in sv.uniq]
            offs = np.zeros(len(enc) + 1, np.int64)
            if enc:
                offs[1:] = np.cumsum([len(b) for b in enc])
            blob = ctypes.create_string_buffer(b"".join(enc), max(int(offs[-1]), 1))
            idx = np.ascontiguousarray(sv.idx, dtype=np.int32)
            keep += [offs, blob, idx]
            f.kind, f.ndims = KIND_STRVEC, 1
            f.dims[0] = idx.size
            f.data = idx.ctypes.data if idx.size else None
            f.blob, f.uniq_off, f.nuniq = ctypes.addressof(blob), offs.ctypes.data, len(enc)
        else:
            raise R2MError(R2M_EINVAL, f"field {name}: unsupported value type {type(v).__name__}")
    check(lib().r2m_jlbin_write(path.encode(), arr, n))


def is_julia_stream(path) -> bool:
    with open(path, "rb") as f:
        return f.read(3) == JULIA_MAGIC
