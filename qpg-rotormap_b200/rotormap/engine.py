"""fp8 search engine (mirror of RotorMap/search/engine_fp8.jl and engine_compact.jl).

TopKEngine wraps the library's fused tcgen05 GEMM + top-k engine
(r2m_engine_*).  The reference's chunk width `w`, top-k segments `segs` and
double-buffered C chunks have no counterpart: scores never leave TMEM.
"""
from __future__ import annotations

import ctypes
from collections.abc import Sequence
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import Tuning, check, lib, ptr, stream_handle
from .encoder import RopeEncoder, encode_frag_real_batch, f16_to_f8
from .fasta import DeviceFastaFragments, FastaFragments, fasta_chunks_device, fasta_reads

_MODES = {"f16": _lib.SCORE_F16, "f32": _lib.SCORE_F32, "scaled": _lib.SCORE_SCALED}
# epilogue form of the fused kernels: auto, 4 warps, or 8 warps (two column
# halves; k <= 32)
_EPILOGUES = {"auto": 0, "4": 1, "8": 2}
# fused kernel variant: one CTA per 128-read tile, or CTA pairs (cta_group::2)
# per 256-read tile; "auto" uses pairs above 128 reads
_KERNELS = {"auto": 0, "1sm": 1, "2sm": 2}


@dataclass
class TopKBatch:
    """One batch of results (engine_fp8.jl:265-271): vals (nb, k) float32
    descending, locs (nb, k) int32 1-based global column ids, norms (nb, m),
    heads (a sequence of strings), first (1-based global index of the batch's
    first read)."""
    vals: np.ndarray
    locs: np.ndarray
    norms: np.ndarray
    heads: Sequence
    first: int


def padmul() -> int:
    """Batch-height multiple of the engine (padmul, engine_fp8.jl:275): the
    fused kernel takes any height, so 1."""
    return 1


class TopKEngine:
    """TopKEngine(B; k, rows_cap, ...) (engine_fp8.jl:290-337).

    B: (N, rdim) uint8 e4m3 CUDA tensor (the reference's (rdim, N)
    column-major embeds8).  score: "f16" (reference cout = :f16, default),
    "f32" (cout = :f32) or "scaled" (per-row / per-column fp32 scales; needs
    scaleB).  The engine owns an e4m3 staging buffer `a8` (rows_cap, rdim) and
    its split workspace; B and the outputs belong to the caller.
    """

    def __init__(self, B: torch.Tensor, k: int = 20, w: int | None = None, rows_cap: int = 8192,
                 segs: int | None = None, score: str = "f16", scaleB: torch.Tensor | None = None,
                 splits: int = 0, ctas: int = 0, timing: bool = False, kernel: str = "auto",
                 epilogue: str = "auto", pace: int = 0, kt: int = 0):
        _lib.require_device()
        if B.dtype != torch.uint8 or B.dim() != 2 or not B.is_cuda or not B.is_contiguous():
            raise ValueError("B must be a contiguous (N, rdim) uint8 CUDA tensor")
        N, rdim = B.shape
        if not (1 <= k <= N):
            raise ValueError(f"need 1 <= k <= N (got k = {k}, N = {N})")
        if score not in _MODES:
            raise ValueError("score must be 'f16', 'f32' or 'scaled'")
        if rdim % 16:
            raise ValueError(f"rdim must be a multiple of 16 (got {rdim})")
        self.B, self.k, self.rows_cap, self.score = B, k, rows_cap, score
        self.scaleB = scaleB
        self.N, self.rdim = N, rdim
        self.a8 = torch.zeros((rows_cap, rdim), dtype=torch.uint8, device=B.device)
        self.scaleA = torch.ones((rows_cap,), dtype=torch.float32, device=B.device)
        if kernel not in _KERNELS:
            raise ValueError("kernel must be 'auto', '1sm' or '2sm'")
        if epilogue not in _EPILOGUES:
            raise ValueError("epilogue must be 'auto', '4' or '8'")
        tune = Tuning(splits, ctas)
        tune.reserved[0] = 1 if timing else 0
        tune.reserved[1] = _KERNELS[kernel]
        tune.reserved[2] = _EPILOGUES[epilogue]
        tune.reserved[3] = int(pace)
        tune.reserved[4] = int(kt)
        self.kernel, self.epilogue, self.pace, self.kt = kernel, epilogue, int(pace), int(kt)
        h = ctypes.c_void_p()
        check(lib().r2m_engine_create(ptr(B), ptr(scaleB), rdim, N, k, rows_cap, _MODES[score],
                                      ctypes.byref(tune), ctypes.byref(h)))
        self._h = h

    @property
    def device(self) -> torch.device:
        return self.B.device

    def set_tuning(self, splits: int = 0, ctas: int = 0, kernel: str | None = None,
                   epilogue: str | None = None, pace: int | None = None, kt: int | None = None) -> None:
        """Change the schedule (0 = automatic; pace: 0 default pacing window,
        > 0 window in column tiles, < 0 off; kt: top-k reservoir size, 0 auto,
        else 8/16/20/32/64 >= k).  Not during stream capture."""
        kernel = kernel or self.kernel
        epilogue = epilogue or self.epilogue
        pace = self.pace if pace is None else int(pace)
        kt = self.kt if kt is None else int(kt)
        if epilogue not in _EPILOGUES:
            raise ValueError("epilogue must be 'auto', '4' or '8'")
        if kernel not in _KERNELS:
            raise ValueError("kernel must be 'auto', '1sm' or '2sm'")
        t = Tuning(splits, ctas)
        t.reserved[1] = _KERNELS[kernel]
        t.reserved[2] = _EPILOGUES[epilogue]
        t.reserved[3] = pace
        t.reserved[4] = kt
        check(lib().r2m_engine_set_tuning(self._h, ctypes.byref(t)))
        self.splits, self.ctas, self.kernel, self.epilogue, self.pace, self.kt = (splits, ctas, kernel, epilogue,
                                                                                  pace, kt)

    def kernel_ms(self):
        """(gemm_ms, merge_ms, splits) of the last search (timing engines only)."""
        g, m, sp = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
        check(lib().r2m_engine_kernel_ms(self._h, ctypes.byref(g), ctypes.byref(m), ctypes.byref(sp)))
        return g.value, m.value, sp.value

    @property
    def workspace_bytes(self) -> int:
        return int(lib().r2m_engine_workspace_bytes(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().r2m_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def search(self, A8: torch.Tensor, nb: int | None = None, scaleA: torch.Tensor | None = None,
               D_val: torch.Tensor | None = None, D_loc: torch.Tensor | None = None, stream=None):
        """Top-k of rows 0..nb-1 of A8 against B -> (D_val (nb, k), D_loc (nb, k))."""
        nb = A8.shape[0] if nb is None else nb
        if nb > self.rows_cap:
            raise ValueError(f"batch height {nb} > engine rows_cap {self.rows_cap}")
        if A8.dtype != torch.uint8 or A8.shape[1] != self.rdim or not A8.is_contiguous():
            raise ValueError("A8 must be a contiguous (nb, rdim) uint8 tensor")
        if self.score == "scaled" and scaleA is None:
            raise ValueError("scaled scores need scaleA")
        dev = self.B.device
        if D_val is None:
            D_val = torch.empty((nb, self.k), dtype=torch.float32, device=dev)
        if D_loc is None:
            D_loc = torch.empty((nb, self.k), dtype=torch.int32, device=dev)
        check(lib().r2m_batch_gemm_topk(self._h, ptr(A8), ptr(scaleA), nb, ptr(D_val), ptr(D_loc),
                                        stream_handle(stream)))
        return D_val, D_loc


class PlainEngine:
    """The plain batch path: the reference engine's structure on the GPU
    (cuBLASLt fp8 GEMM into fp16 chunks of `w` columns + segmented top-k,
    engine_fp8.jl:290-437).  Same search() contract as TopKEngine for
    score = "f16"; ties follow the reference's segment/reservoir order."""

    def __init__(self, B: torch.Tensor, k: int = 20, w: int = 65536, rows_cap: int = 8192, segs: int = 8):
        _lib.require_device()
        if B.dtype != torch.uint8 or B.dim() != 2 or not B.is_cuda or not B.is_contiguous():
            raise ValueError("B must be a contiguous (N, rdim) uint8 CUDA tensor")
        self.B, self.k, self.N, self.rdim = B, k, B.shape[0], B.shape[1]
        self.w = min(w, self.N)
        self.rows_cap = (rows_cap + 15) // 16 * 16
        self.score = "f16"
        self.a8 = torch.zeros((self.rows_cap, self.rdim), dtype=torch.uint8, device=B.device)
        h = ctypes.c_void_p()
        check(lib().r2m_plain_engine_create(ptr(B), self.rdim, self.N, k, self.rows_cap, self.w, segs,
                                            ctypes.byref(h)))
        self._h = h

    @property
    def device(self) -> torch.device:
        return self.B.device

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().r2m_plain_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def search(self, A8: torch.Tensor, nb: int | None = None, scaleA=None, D_val=None, D_loc=None,
               stream=None):
        """A8 must hold ceil(nb/16)*16 rows (use the engine's `a8` staging)."""
        nb = A8.shape[0] if nb is None else nb
        if nb > self.rows_cap or A8.shape[0] < (nb + 15) // 16 * 16:
            raise ValueError("A8 must hold ceil(nb/16)*16 rows within rows_cap")
        dev = self.B.device
        if D_val is None:
            D_val = torch.empty((nb, self.k), dtype=torch.float32, device=dev)
        if D_loc is None:
            D_loc = torch.empty((nb, self.k), dtype=torch.int32, device=dev)
        check(lib().r2m_plain_batch_gemm_topk(self._h, ptr(A8), nb, ptr(D_val), ptr(D_loc),
                                              stream_handle(stream)))
        return D_val, D_loc


class CompactEngine:
    """CompactEngine(host; k, rows_cap, ...) (engine_compact.jl:256-289): the
    index stays in host memory -- a C-contiguous (N, rdim) uint8 numpy array
    (a memory-mapped index file works) or a CPU uint8 tensor -- and each
    search streams it through `depth` device slots of about `chunk_cols`
    columns.  Same search() contract and the same results, bit for bit, as
    TopKEngine over the whole index.  resident_chunks leading chunks get
    device slots of their own, copied once ("auto": as many as the free
    device memory holds beside the ring and a 2 GiB reserve), so only the
    rest crosses the host link on every search.  pin page-locks the host
    index for the engine's lifetime (full-speed DMA; refused registrations
    stay pageable).  scaleB (scaled scores) is uploaded once (4 bytes per
    column)."""

    def __init__(self, Bh, k: int = 20, rows_cap: int = 8192, score: str = "f16", scaleB=None,
                 chunk_cols: int = 1 << 20, depth: int = 3, pin: bool = True, device=None, splits: int = 0,
                 ctas: int = 0, kernel: str = "auto", resident_chunks=0):
        _lib.require_device()
        if isinstance(Bh, torch.Tensor):
            if Bh.is_cuda or Bh.dtype != torch.uint8 or Bh.dim() != 2:
                raise ValueError("a tensor host index must be a 2-D uint8 CPU tensor")
            Bh = Bh.contiguous()
            addr = Bh.data_ptr()
        else:
            Bh = np.asarray(Bh)
            if Bh.dtype != np.uint8 or Bh.ndim != 2:
                raise ValueError("the host index must be a 2-D uint8 array")
            if not Bh.flags.c_contiguous:
                Bh = np.ascontiguousarray(Bh)
            addr = Bh.ctypes.data
        N, rdim = Bh.shape
        if score not in _MODES:
            raise ValueError("score must be 'f16', 'f32' or 'scaled'")
        if kernel not in _KERNELS:
            raise ValueError("kernel must be 'auto', '1sm' or '2sm'")
        self.host, self.k, self.rows_cap, self.score = Bh, k, rows_cap, score
        self.N, self.rdim = int(N), int(rdim)
        self._device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.scaleB = None
        if score == "scaled":
            if scaleB is None:
                raise ValueError("scaled scores need scaleB")
            sb = scaleB if isinstance(scaleB, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(scaleB))
            self.scaleB = sb.to(self._device, torch.float32).contiguous()
        self.a8 = torch.zeros((rows_cap, rdim), dtype=torch.uint8, device=self._device)
        self.scaleA = torch.ones((rows_cap,), dtype=torch.float32, device=self._device)
        tune = Tuning(splits, ctas)
        tune.reserved[1] = _KERNELS[kernel]
        if resident_chunks == "auto":
            resident_chunks = self.auto_resident_chunks(self.N, rdim, chunk_cols, depth, self._device)
        if int(resident_chunks) < 0:
            raise ValueError("resident_chunks must be >= 0 or 'auto'")
        h = ctypes.c_void_p()
        with torch.cuda.device(self._device):
            check(lib().r2m_compact_create(addr, ptr(self.scaleB), self.rdim, self.N, k, rows_cap, _MODES[score],
                                           chunk_cols, depth, int(resident_chunks), 1 if pin else 0,
                                           ctypes.byref(tune), ctypes.byref(h)))
        self._h = h

    @staticmethod
    def auto_resident_chunks(N: int, rdim: int, chunk_cols: int, depth: int, device=None,
                             reserve: int = 2 << 30) -> int:
        """Chunks that fit in the device memory free now beside the ring's
        `depth` slots and `reserve` bytes."""
        nch = -(-N // chunk_cols)
        slot = (-(-N // nch) + 4) * rdim
        free, _ = torch.cuda.mem_get_info(device)
        return int(max(0, min(nch, (free - reserve - depth * slot) // slot)))

    @property
    def resident_chunks(self) -> int:
        return int(lib().r2m_compact_resident_chunks(self._h))

    @property
    def device(self) -> torch.device:
        return self._device

    @property
    def chunks(self) -> int:
        return int(lib().r2m_compact_chunks(self._h))

    @property
    def pinned(self) -> bool:
        return bool(lib().r2m_compact_is_pinned(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().r2m_compact_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def search(self, A8: torch.Tensor, nb: int | None = None, scaleA: torch.Tensor | None = None,
               D_val: torch.Tensor | None = None, D_loc: torch.Tensor | None = None, stream=None):
        """batch_gemm_topk_compact! (engine_compact.jl:300-343): top-k of rows
        0..nb-1 of A8 against the host index -> (D_val (nb, k), D_loc (nb, k))."""
        nb = A8.shape[0] if nb is None else nb
        if nb > self.rows_cap:
            raise ValueError(f"batch height {nb} > engine rows_cap {self.rows_cap}")
        if A8.dtype != torch.uint8 or A8.shape[1] != self.rdim or not A8.is_contiguous():
            raise ValueError("A8 must be a contiguous (nb, rdim) uint8 tensor")
        if self.score == "scaled" and scaleA is None:
            raise ValueError("scaled scores need scaleA")
        dev = self._device
        if D_val is None:
            D_val = torch.empty((nb, self.k), dtype=torch.float32, device=dev)
        if D_loc is None:
            D_loc = torch.empty((nb, self.k), dtype=torch.int32, device=dev)
        check(lib().r2m_compact_batch_gemm_topk(self._h, ptr(A8), ptr(scaleA), nb, ptr(D_val), ptr(D_loc),
                                                stream_handle(stream)))
        return D_val, D_loc


def upload_fp16_as_f8(eng: TopKEngine, embeds, stream=None) -> torch.Tensor:
    """upload_fp16_as_f8! (engine_fp8.jl:355-371): H2D an fp16 (nb, rdim) batch
    and quantise it into the engine staging `a8` rows 0..nb-1."""
    e = torch.as_tensor(embeds)
    if e.dtype != torch.float16:
        raise TypeError("embeds must be float16")
    nb, rdim = e.shape
    if rdim != eng.rdim or nb > eng.rows_cap:
        raise ValueError("batch shape does not fit the engine staging")
    d = e.to(eng.device, non_blocking=True).contiguous()
    f16_to_f8(eng.a8[:nb], d, stream)
    return eng.a8


def batch_gemm_topk(D_val: torch.Tensor, D_loc: torch.Tensor, eng: TopKEngine, nb: int | None = None,
                    A8: torch.Tensor | None = None, scaleA: torch.Tensor | None = None, stream=None):
    """batch_gemm_topk! (engine_fp8.jl:399-437): top-k of the staged batch
    (eng.a8 unless A8 is given) into D_val / D_loc (at least nb rows)."""
    A = eng.a8 if A8 is None else A8
    nb = A.shape[0] if nb is None else nb
    sa = scaleA if scaleA is not None else (eng.scaleA if eng.score == "scaled" else None)
    eng.search(A, nb, sa, D_val, D_loc, stream)
    return D_val, D_loc


class Mapper:
    """Batch mapping through the public API with host buffers: packed read
    words (host) -> H2D -> fused encode -> fp8 GEMM + top-k -> D2H of the
    (nb, k) results.  Pinned staging is allocated once for `rows_cap` reads."""

    def __init__(self, eng: TopKEngine, re: RopeEncoder, normalize: int = 0, stream=None):
        self.eng, self.re, self.normalize = eng, re, normalize
        dev = eng.device
        cap = eng.rows_cap
        self.stream = stream or torch.cuda.Stream(dev)
        self.h_words = torch.empty((cap, re.words), dtype=torch.int32, pin_memory=True)
        self.h_vals = torch.empty((cap, eng.k), dtype=torch.float32, pin_memory=True)
        self.h_locs = torch.empty((cap, eng.k), dtype=torch.int32, pin_memory=True)
        self.d_words = torch.empty((cap, re.words), dtype=torch.int32, device=dev)
        self.d_norms = torch.empty((cap, re.m), dtype=torch.float32, device=dev)
        self.d_vals = torch.empty((cap, eng.k), dtype=torch.float32, device=dev)
        self.d_locs = torch.empty((cap, eng.k), dtype=torch.int32, device=dev)

    def h2d_bytes(self, nb: int) -> int:
        return nb * self.re.words * 4

    def d2h_bytes(self, nb: int) -> int:
        return nb * self.eng.k * 8

    def map_words(self, words: np.ndarray | None = None, nb: int | None = None):
        """Map `nb` reads whose packed words are in `words` (or already in
        self.h_words).  Returns host views (vals (nb, k), locs (nb, k))."""
        if words is not None:
            nb = words.shape[0]
            self.h_words[:nb].numpy().view(np.uint32)[:] = words
        eng, st = self.eng, self.stream
        scaled = eng.score == "scaled"
        with torch.cuda.stream(st):
            self.d_words[:nb].copy_(self.h_words[:nb], non_blocking=True)
            a8 = eng.a8[:nb]
            sa = eng.scaleA[:nb] if scaled else None
            encode_frag_real_batch(a8, self.d_norms[:nb], self.re, self.d_words[:nb], self.normalize, sa, st)
            eng.search(a8, nb, sa, self.d_vals[:nb], self.d_locs[:nb], st)
            self.h_vals[:nb].copy_(self.d_vals[:nb], non_blocking=True)
            self.h_locs[:nb].copy_(self.d_locs[:nb], non_blocking=True)
        st.synchronize()
        return self.h_vals[:nb].numpy(), self.h_locs[:nb].numpy()


# ------------------------------------------------------------------ flows


def _batches(frags: FastaFragments | DeviceFastaFragments, batch_size: int):
    for b0 in range(0, len(frags), batch_size):
        yield b0, frags.words[b0:b0 + batch_size], frags.heads[b0:b0 + batch_size]


def _chunked_batches(pieces, batch_size: int):
    """Batches over consecutive reader pieces, numbered across the input."""
    first0 = 0
    for frags in pieces:
        for b0, words, heads in _batches(frags, batch_size):
            yield first0 + b0, words, heads
        first0 += len(frags)


def topk_flow(source, eng: TopKEngine, re: RopeEncoder, normalize: int = 0, stream=None):
    """topk_flow (engine_fp8.jl:498-547) over an iterable of
    (first0, words (nb, W), heads) batches -- words as host uint32 arrays or
    as int32 CUDA tensors already on the engine's device: encode on the GPU
    straight to e4m3 (fp16-rounded, or per-row scaled for score = "scaled"),
    search, and yield TopKBatch with host arrays."""
    dev = eng.device
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    scaled = eng.score == "scaled"
    for first0, words, heads in source:
        nb = words.shape[0]
        if nb == 0:
            continue
        if nb > eng.rows_cap:
            raise ValueError(f"batch height {nb} > engine rows_cap {eng.rows_cap}")
        on_device = isinstance(words, torch.Tensor) and words.is_cuda
        if not on_device:
            hw = torch.from_numpy(np.ascontiguousarray(words, dtype=np.uint32)).pin_memory()
        with torch.cuda.stream(st):
            if on_device:
                dw = words.contiguous()
            else:
                dw = hw.to(dev, non_blocking=True).view(torch.int32)
            norms = torch.empty((nb, re.m), dtype=torch.float32, device=dev)
            a8 = eng.a8[:nb]
            sa = eng.scaleA[:nb] if scaled else None
            encode_frag_real_batch(a8, norms, re, dw, normalize, sa, st)
            D_val, D_loc = eng.search(a8, nb, sa, stream=st)
            vals = D_val.to("cpu", non_blocking=True)
            locs = D_loc.to("cpu", non_blocking=True)
            nrm = norms.to("cpu", non_blocking=True)
        st.synchronize()
        yield TopKBatch(vals.numpy(), locs.numpy(), nrm.numpy(), heads, first0 + 1)


HOST_READER_MAX_BYTES = 8 << 30  # inputs the host reader takes whole


def pick_reader(file, reader: str = "auto") -> str:
    """reader = "auto" (the flows' default): the native host reader when the
    host has >= 8 threads and the input is at most 8 GiB (it parses the
    whole input at once), else the GPU reader, which streams any input size
    through bounded memory.  Parsing alone from host bytes the host reader
    is faster (6.3 vs 3.9 GB/s on 16 threads); in the whole run_map flow,
    where host threads also format the table, the two are within a few
    percent of each other (514K vs 512K reads/s in one run, 459K vs 517K in
    another, same box)."""
    if reader != "auto":
        return reader
    import os
    if isinstance(file, (bytes, bytearray, memoryview)):
        size = len(file)
    else:
        try:
            size = os.path.getsize(file)
        except (OSError, TypeError):
            return "device"
    return "host" if (os.cpu_count() or 1) >= 8 and size <= HOST_READER_MAX_BYTES else "device"


def rope_topk_stream(re: RopeEncoder, file, B: torch.Tensor, k: int = 20, w: int | None = None,
                     batch_size: int = 8192, rows_cap: int | None = None, normalize: int = 0,
                     score: str = "f16", scaleB: torch.Tensor | None = None, parts: int | None = None,
                     segs: int | None = None, engine: TopKEngine | None = None, stream=None,
                     reader: str = "auto", chunk_bytes: int = 1 << 30):
    """rope_topk_stream (engine_fp8.jl:576-594): FASTA -> encode -> fp8 GEMM +
    top-k against the resident B -> TopKBatch per batch (file order).

    reader = "device" (the default) parses the FASTA on the GPU (the words stay in HBM),
    `chunk_bytes` of the file at a time (cut at record starts), so inputs of
    any size stream through bounded memory; "host" uses the native host
    reader with `parts` threads on the whole input.  Both give the same
    reads."""
    if B.shape[1] != re.rdim:
        raise ValueError(f"B is {tuple(B.shape)}; the encoder's real embedding dim is {re.rdim}")
    reader = pick_reader(file, reader)
    if reader == "device":
        source = _chunked_batches(fasta_chunks_device(file, k=re.k, chunk_bytes=chunk_bytes, device=B.device,
                                                      stream=stream), batch_size)
    elif reader == "host":
        source = _batches(fasta_reads(file, k=re.k, parts=parts), batch_size)
    else:
        raise ValueError('reader must be "auto", "device" or "host"')
    eng = engine or TopKEngine(B, k=k, rows_cap=rows_cap or batch_size, score=score, scaleB=scaleB)
    yield from topk_flow(source, eng, re, normalize, stream)


def resident_need(host_bytes: int, rows_cap: int, rdim: int, k: int = 20) -> int:
    """_resident_need (engine_compact.jl:195-205) for this engine: B + the e4m3
    staging + per-batch temps + the split workspace bound + slack."""
    return int(host_bytes + rows_cap * rdim * 2 + rows_cap * 64 * k * 8 * 2 + 96 * 2 ** 20)


def resident_fits(host_bytes: int, rows_cap: int, rdim: int, k: int = 20, device=None) -> bool:
    """resident_fits (engine_compact.jl:238-242): the index plus the engine's
    working set fits the device memory free right now."""
    free, _ = torch.cuda.mem_get_info(device)
    return resident_need(host_bytes, rows_cap, rdim, k) <= free


def rope_topk_stream_compact(re: RopeEncoder, file, Bh, k: int = 20, batch_size: int = 8192,
                             rows_cap: int | None = None, normalize: int = 0, score: str = "f16",
                             scaleB=None, resident: bool | None = None, chunk_cols: int = 1 << 20,
                             depth: int = 3, pin: bool = True, reader: str = "auto", parts: int | None = None,
                             stream=None, resident_chunks="auto"):
    """rope_topk_stream_compact (engine_compact.jl:415-457) with a host index
    Bh (N, rdim) uint8.  resident = None applies resident_fits: an index that
    fits beside the engine's working set is uploaded once and searched by
    the resident engine; otherwise (or resident = False) it stays in host
    memory and the CompactEngine keeps resident_chunks of it on the device
    ("auto": as many as fit) and streams the rest through its ring for every
    batch.  Both give the same batches."""
    Bh = np.asarray(Bh) if not isinstance(Bh, torch.Tensor) else Bh
    nbytes = Bh.nbytes if isinstance(Bh, np.ndarray) else Bh.numel()
    cap = rows_cap or batch_size
    if resident is None:
        resident = resident_fits(nbytes, cap, re.rdim, k)
    sb = None
    if scaleB is not None:
        sb = scaleB if isinstance(scaleB, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(scaleB))
        sb = sb.cuda()
    if resident:
        if isinstance(Bh, torch.Tensor):
            B = Bh if Bh.is_cuda else Bh.cuda()
        else:
            B = torch.from_numpy(np.ascontiguousarray(Bh)).cuda()
        yield from rope_topk_stream(re, file, B, k=k, batch_size=batch_size, rows_cap=cap, normalize=normalize,
                                    score=score, scaleB=sb, reader=reader, parts=parts, stream=stream)
        return
    if Bh.shape[1] != re.rdim:
        raise ValueError(f"B is {tuple(Bh.shape)}; the encoder's real embedding dim is {re.rdim}")
    eng = CompactEngine(Bh, k=k, rows_cap=cap, score=score, scaleB=sb, chunk_cols=chunk_cols, depth=depth,
                        pin=pin, resident_chunks=resident_chunks)
    try:
        reader = pick_reader(file, reader)
        if reader == "device":
            source = _chunked_batches(fasta_chunks_device(file, k=re.k, device=eng.device, stream=stream),
                                      batch_size)
        elif reader == "host":
            source = _batches(fasta_reads(file, k=re.k, parts=parts), batch_size)
        else:
            raise ValueError('reader must be "auto", "device" or "host"')
        yield from topk_flow(source, eng, re, normalize, stream)
    finally:
        eng.close()
