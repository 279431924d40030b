"""FASTA reads -> forward 2-bit words (mirror of RotorMap/fasta/reader.jl).

Parsing runs in the library's native C++ reader (r2m_fasta_reads); this
module only moves its result into numpy.
"""
from __future__ import annotations

import ctypes
import mmap
import os
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib


@dataclass
class FastaFragments:
    """All kept records: words (n, cld(k,16)) uint32, verbatim '>' headers."""
    k: int
    words: np.ndarray
    heads: list

    def __len__(self) -> int:
        return len(self.heads)


def _read_bytes(src) -> bytes | mmap.mmap:
    if isinstance(src, (bytes, bytearray, memoryview)):
        return bytes(src)
    path = os.fspath(src)
    if os.path.getsize(path) == 0:
        return b""
    with open(path, "rb") as f:
        return mmap.mmap(f.fileno(), 0, access=mmap.ACCESS_READ)


def fasta_reads(src, k: int = 20_000, parts: int | None = None) -> FastaFragments:
    """fasta_reads(file; k, parts) (RotorMap/fasta/reader.jl:321-350).

    Every record is trimmed to its first k bases; records with fewer bases
    are skipped; unknown bytes become G.  Returns records in file order.
    """
    if k < 1:
        raise ValueError("k must be >= 1")
    data = _read_bytes(src)
    n = len(data)
    if isinstance(data, mmap.mmap):
        buf = (ctypes.c_char * n).from_buffer_copy(data) if n else b""
        data.close()
    else:
        buf = data
    handle = ctypes.c_void_p()
    L = lib()
    nthreads = parts if parts else (os.cpu_count() or 1)
    check(L.r2m_fasta_reads(buf, n, k, nthreads, ctypes.byref(handle)))
    try:
        cnt = L.r2m_reads_count(handle)
        W = (k + 15) // 16
        if cnt:
            wp = L.r2m_reads_words(handle)
            words = np.ctypeslib.as_array((ctypes.c_uint32 * (cnt * W)).from_address(wp)).copy()
            words = words.reshape(cnt, W)
        else:
            words = np.zeros((0, W), np.uint32)
        heads = []
        ln = ctypes.c_size_t()
        for i in range(cnt):
            p = L.r2m_reads_header(handle, i, ctypes.byref(ln))
            heads.append(ctypes.string_at(p, ln.value).decode("latin-1"))
    finally:
        L.r2m_reads_free(handle)
    return FastaFragments(k, words, heads)
