"""FASTA reads -> forward 2-bit words (mirror of RotorMap/fasta/reader.jl).

Two readers with the same result: fasta_reads parses on the host in the
library's native C++ reader (r2m_fasta_reads) and returns numpy words;
fasta_reads_device uploads the FASTA bytes and parses them on the GPU
(r2m_fasta_reads_device), leaving the words in HBM for the encoder.
"""
from __future__ import annotations

import ctypes
import mmap
import os
import threading
from collections.abc import Sequence
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib, ptr, require_device, stream_handle


class HeaderList(Sequence):
    """Read headers kept as one blob (every header followed by '\n'; headers
    hold no '\n') with their start offsets: an item is decoded when it is
    read, a slice is a view of the same blob, and the list compares equal to
    a list of the same strings.  The table writer takes the blob as is."""

    __slots__ = ("_blob", "_off")

    def __init__(self, blob: bytes, offsets):
        self._blob = blob
        self._off = np.asarray(offsets, np.int64)  # n + 1 offsets; header i ends at off[i + 1] - 1

    @classmethod
    def from_blob(cls, blob: bytes) -> "HeaderList":
        ends = np.flatnonzero(np.frombuffer(blob, np.uint8) == 0x0A)
        return cls(blob, np.concatenate([[0], ends + 1]))

    def __len__(self) -> int:
        return self._off.size - 1

    def __getitem__(self, i):
        n = len(self)
        if isinstance(i, slice):
            start, stop, step = i.indices(n)
            if step != 1:
                return [self[j] for j in range(start, stop, step)]
            stop = max(stop, start)
            return HeaderList(self._blob, self._off[start:stop + 1])
        if i < 0:
            i += n
        if not 0 <= i < n:
            raise IndexError("header index out of range")
        return self._blob[self._off[i]:self._off[i + 1] - 1].decode("latin-1")

    def __iter__(self):
        if len(self) == 0:
            return iter(())
        return iter(self.blob().decode("latin-1").split("\n")[:-1])

    def blob(self) -> bytes:
        """The headers of this list, each followed by '\n'."""
        if len(self) == 0:
            return b""
        return self._blob[self._off[0]:self._off[-1]]

    def __eq__(self, other):
        if isinstance(other, (list, tuple, HeaderList)):
            return list(self) == list(other)
        return NotImplemented

    def __repr__(self) -> str:
        return f"HeaderList({len(self)} headers)"


@dataclass
class FastaFragments:
    """All kept records: words (n, cld(k,16)) uint32, verbatim '>' headers."""
    k: int
    words: np.ndarray
    heads: Sequence

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
    keep = None
    if isinstance(data, mmap.mmap):
        # parse straight from the mapping (no copy of the file)
        keep = np.frombuffer(data, np.uint8)
        buf = ctypes.c_char_p(keep.ctypes.data)
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
        heads = HeaderList(b"", [0])
        if cnt:
            tot = ctypes.c_size_t()
            bp = L.r2m_reads_header_blob(handle, ctypes.byref(tot))
            op = L.r2m_reads_header_offsets(handle)
            offs = np.ctypeslib.as_array((ctypes.c_size_t * (cnt + 1)).from_address(op)).astype(np.int64)
            heads = HeaderList(ctypes.string_at(bp, tot.value), offs)
    finally:
        L.r2m_reads_free(handle)
        if keep is not None:
            del keep
            data.close()
    return FastaFragments(k, words, heads)


@dataclass
class DeviceFastaFragments:
    """Kept records parsed on the GPU: words (n, cld(k,16)) int32 on the
    device (the uint32 bit pattern), verbatim '>' headers on the host."""
    k: int
    words: "torch.Tensor"
    heads: Sequence
    stopped: bool = False  # an unclosed header ended the parse

    def __len__(self) -> int:
        return len(self.heads)


_PINNED = threading.local()


def _pinned(tag: str, nbytes: int):
    """A grow-only pinned host buffer per tag and thread (the caller
    synchronises its stream before the buffer is reused)."""
    import torch
    bufs = getattr(_PINNED, "bufs", None)
    if bufs is None:
        bufs = _PINNED.bufs = {}
    buf = bufs.get(tag)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, pin_memory=True)
        bufs[tag] = buf
    return buf[:nbytes]


def fasta_reads_device(src, k: int = 20_000, device=None, stream=None) -> DeviceFastaFragments:
    """fasta_reads on the GPU: the same records, words and headers.

    src is FASTA bytes, a path, or a uint8 CUDA tensor already holding the
    bytes.  Host sources are staged through a reused pinned buffer and
    copied to the device on `stream`; the parse runs there; the headers come
    back as one blob ('\n' after each) and are split on the host.
    """
    import torch

    if k < 1:
        raise ValueError("k must be >= 1")
    require_device()
    if isinstance(src, torch.Tensor):
        if not src.is_cuda or src.dtype != torch.uint8:
            raise ValueError("a tensor source must be a uint8 CUDA tensor")
        dev_bytes = src.contiguous().view(-1)
        dev = dev_bytes.device
        host = None
    else:
        host = None
        if not isinstance(src, (bytes, bytearray, memoryview)):
            path = os.fspath(src)
            size = os.path.getsize(path)
        else:
            host = np.frombuffer(src, np.uint8) if len(src) else np.zeros(0, np.uint8)
            size = host.size
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        dev_bytes = None
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    L = lib()
    with torch.cuda.device(dev), torch.cuda.stream(st):
        if dev_bytes is None:
            stage = _pinned("fasta_in", size)
            if size:
                if host is not None:
                    stage.numpy()[:] = host
                else:  # read the file straight into the pinned buffer
                    with open(path, "rb") as f:
                        got = f.readinto(memoryview(stage.numpy()))
                    if got != size:
                        raise OSError(f"short read of {path}: {got} of {size} bytes")
            dev_bytes = stage.to(dev, non_blocking=True)
        handle = ctypes.c_void_p()
        n = int(dev_bytes.numel())
        check(L.r2m_fasta_reads_device(ptr(dev_bytes) if n else None, n, k, stream_handle(st), ctypes.byref(handle)))
        try:
            cnt = int(L.r2m_dreads_count(handle))
            stopped = bool(L.r2m_dreads_stopped(handle))
            W = (k + 15) // 16
            words = torch.empty((cnt, W), dtype=torch.int32, device=dev)
            heads = HeaderList(b"", [0])
            if cnt:
                words.view(-1).copy_(_wrap_device(L.r2m_dreads_words(handle), cnt * W, torch.int32, dev))
                tot = ctypes.c_size_t()
                hp = L.r2m_dreads_header_blob(handle, ctypes.byref(tot))
                hb = _pinned("fasta_heads", tot.value)
                hb.copy_(_wrap_device(hp, tot.value, torch.uint8, dev), non_blocking=True)
                st.synchronize()
                heads = HeaderList.from_blob(hb.numpy().tobytes())
        finally:
            st.synchronize()
            L.r2m_dreads_free(handle)
    return DeviceFastaFragments(k, words, heads, stopped)


def _last_record_start(buf: bytes) -> int:
    """Offset of the last record start after offset 0 (a '>' that follows
    '\n' or '\r'), or -1."""
    i = max(buf.rfind(b"\n>"), buf.rfind(b"\r>"))
    return i + 1 if i >= 0 else -1


def _fasta_pieces(src, chunk_bytes: int):
    """The input (bytes or a path) in pieces of about `chunk_bytes`, each cut
    at its last record start (the rest carries over); a piece that holds no
    record start after its first byte grows until one appears or the input
    ends.  The pieces concatenate to the input and no record spans two."""
    import io as _io
    if chunk_bytes < 1:
        raise ValueError("chunk_bytes must be >= 1")
    f = _io.BytesIO(bytes(src)) if isinstance(src, (bytes, bytearray, memoryview)) else open(os.fspath(src), "rb")
    try:
        carry = b""
        while True:
            block = f.read(chunk_bytes)
            eof = len(block) < chunk_bytes
            data = carry + block if carry else block
            if not eof:
                cut = _last_record_start(data)
                if cut <= 0:  # no record start after the first byte yet: read on
                    carry = data
                    continue
                piece, carry = data[:cut], data[cut:]
            else:
                piece, carry = data, b""
            if piece:
                yield piece
            if eof:
                return
    finally:
        f.close()


def fasta_chunks_device(src, k: int = 20_000, chunk_bytes: int = 1 << 30, device=None, stream=None):
    """fasta_reads on the GPU for inputs of any size: the file (or bytes) is
    read in blocks of about `chunk_bytes`, each cut at its last record start
    (the rest carries over to the next block), and every piece is parsed by
    fasta_reads_device.  Pieces never split a record, so the records, words
    and headers are those of the whole input; after a piece in which an
    unclosed header ended the parse, nothing further is read (the rule of
    the whole-input reader).  Yields DeviceFastaFragments in file order."""
    for piece in _fasta_pieces(src, chunk_bytes):
        frags = fasta_reads_device(piece, k=k, device=device, stream=stream)
        yield frags
        if frags.stopped:
            return


def _wrap_device(addr: int, count: int, dtype, dev):
    """A torch view of `count` elements of library-owned device memory."""
    import torch

    class _Cai:
        __cuda_array_interface__ = {
            "shape": (count,),
            "typestr": {torch.int32: "<i4", torch.int64: "<i8", torch.uint8: "|u1"}[dtype],
            "data": (addr, False),
            "version": 3,
            "strides": None,
        }

    return torch.as_tensor(_Cai(), device=dev)
