"""Index build / save / load (mirror of RotorMap/index/build.jl and load.jl).

The reference index is a Julia-serialized NamedTuple (format
"indexreal.fp8.v1": embeds8 (rdim, 2*n_frag) e4m3 columns, norms (m, 2*n_frag),
heads, starts (1-based), strand (0 fwd / 1 rc), k, kstep, s, m, c,
normalize).  `save_index` writes that file (the library's Serialization
writer, csrc/jlser.cpp) and `load_index` reads it, memory-mapped, with the
reference loader's checks; it also reads the reference's fp16/fp32 row
layout ("indexreal.v1") and the pre-rename format tags.  A second, optional
container (magic "R2MIDX01", a JSON header, 64-byte aligned raw arrays;
files named *.r2mi) also keeps the packed genome that FP32 rescoring
re-encodes windows from, which the reference's NamedTuple does not carry.

Build: the host packs every record once into 2-bit words (each record starts
on a word boundary and is followed by a zero guard word), lists the window
starts (offsets 0, kstep, ... with the window fully inside the record,
build.jl:291-324) and the GPU encodes the forward and reverse-complement
window of every start straight into e4m3 index columns
(r2m_encode_ref_windows), in the reference's per-batch [fwd | rc] column
order (build.jl:640-660).
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_handle
from .encoder import RopeEncoder

FP8_FORMAT = "indexreal.fp8.v1"          # load.jl:31
ROW_FORMAT = "indexreal.v1"              # load.jl:30 (fp16 / fp32 rows)
LEGACY_FP8_FORMAT = "indexflowreal.fp8.v1"  # load.jl:33-34 (pre-rename saves)
LEGACY_ROW_FORMAT = "indexflowreal.v1"
SCALED_FORMAT = "indexreal.fp8scaled.v1"  # per-column scaled e4m3 (precision form)
_MAGIC = b"R2MIDX01"

@dataclass
class RefPack:
    """Packed reference: verbatim headers, per-record word offset / base count."""
    heads: list
    word_off: np.ndarray   # int64, first word of each record in `words`
    nbases: np.ndarray     # int64
    words: np.ndarray      # uint32, all records + guard words


def _pack_codes(codes: np.ndarray) -> np.ndarray:
    n = codes.size
    nw = (n + 15) // 16
    pad = np.zeros(nw * 16, np.uint32)
    pad[:n] = codes
    sh = (2 * np.arange(16, dtype=np.uint32))[None, :]
    return np.bitwise_or.reduce(pad.reshape(nw, 16) << sh, axis=1).astype(np.uint32)


def pack_records(heads, codes_list) -> RefPack:
    """Pack records given as 2-bit code arrays (one per record)."""
    offs, nb, chunks = [], [], []
    cur = 0
    for codes in codes_list:
        codes = np.asarray(codes, dtype=np.uint8)
        w = _pack_codes(codes)
        offs.append(cur)
        nb.append(codes.size)
        chunks.append(w)
        chunks.append(np.zeros(1, np.uint32))  # guard word
        cur += w.size + 1
    words = np.concatenate(chunks) if chunks else np.zeros(1, np.uint32)
    return RefPack(list(heads), np.array(offs, np.int64), np.array(nb, np.int64), words)


def pack_reference(src, nthreads: int | None = None) -> RefPack:
    """Parse a reference FASTA (bytes or a path) and pack every record, in
    the library's native multithreaded packer (r2m_fasta_genome; the record
    walk of build.jl:291-324)."""
    import ctypes
    import mmap
    if isinstance(src, (bytes, bytearray, memoryview)):
        data, keep = bytes(src), None
    else:
        path = os.fspath(src)
        if os.path.getsize(path) == 0:
            data, keep = b"", None
        else:
            with open(path, "rb") as f:
                keep = mmap.mmap(f.fileno(), 0, access=mmap.ACCESS_READ)
            data = None
    L = lib()
    handle = ctypes.c_void_p()
    if keep is not None:
        arr = np.frombuffer(keep, np.uint8)
        addr, n = arr.ctypes.data, arr.size
    else:
        arr = np.frombuffer(data, np.uint8) if data else np.zeros(0, np.uint8)
        addr, n = (arr.ctypes.data if arr.size else None), arr.size
    try:
        check(L.r2m_fasta_genome(addr, n, nthreads or (os.cpu_count() or 1), ctypes.byref(handle)))
    finally:
        del arr
        if keep is not None:
            keep.close()
    try:
        R = int(L.r2m_genome_count(handle))
        nw = ctypes.c_size_t()
        wp = L.r2m_genome_words(handle, ctypes.byref(nw))
        words = np.ctypeslib.as_array((ctypes.c_uint32 * nw.value).from_address(wp)).copy()
        if R:
            off = np.ctypeslib.as_array((ctypes.c_int64 * R).from_address(L.r2m_genome_word_off(handle))).copy()
            nb = np.ctypeslib.as_array((ctypes.c_int64 * R).from_address(L.r2m_genome_nbases(handle))).copy()
            tot = ctypes.c_size_t()
            hp = L.r2m_genome_header_blob(handle, ctypes.byref(tot))
            heads = ctypes.string_at(hp, tot.value).decode("latin-1").split("\n")[:R]
        else:
            off, nb, heads = np.zeros(0, np.int64), np.zeros(0, np.int64), []
    finally:
        L.r2m_genome_free(handle)
    return RefPack(heads, off, nb, words)


def window_positions(pack: RefPack, k: int, kstep: int):
    """Window starts fully inside each record: (pos, rec, start_1based)."""
    pos, rec, st = [], [], []
    for r, (wo, nbases) in enumerate(zip(pack.word_off, pack.nbases)):
        if nbases < k:
            continue
        offs = np.arange(0, nbases - k + 1, kstep, dtype=np.int64)
        pos.append(16 * wo + offs)
        rec.append(np.full(offs.size, r, np.int32))
        st.append(offs + 1)
    if not pos:
        return np.zeros(0, np.int64), np.zeros(0, np.int32), np.zeros(0, np.int64)
    return np.concatenate(pos), np.concatenate(rec), np.concatenate(st)


def batch_column_order(nwin: int, batch: int):
    """Column -> (window, strand) under the per-batch [fwd block | rc block] layout."""
    col_win = np.empty(2 * nwin, np.int64)
    strand = np.empty(2 * nwin, np.uint8)
    for b0 in range(0, nwin, batch):
        nb = min(batch, nwin - b0)
        c0 = 2 * b0
        w = np.arange(b0, b0 + nb, dtype=np.int64)
        col_win[c0:c0 + nb] = w
        col_win[c0 + nb:c0 + 2 * nb] = w
        strand[c0:c0 + nb] = 0
        strand[c0 + nb:c0 + 2 * nb] = 1
    return col_win, strand


@dataclass
class Index:
    """The loaded/built index: reference NamedTuple fields + packed genome."""
    format: str
    source: str
    k: int
    kstep: int
    s: int
    m: int
    c: int
    normalize: int
    n_frag: int
    embeds8: object            # (N, rdim) uint8: torch CUDA tensor or numpy (host)
    norms: np.ndarray          # (N, m) float32
    rec_heads: list            # unique record headers (verbatim, with '>')
    col_rec: np.ndarray        # (N,) int32 record of each column
    starts: np.ndarray         # (N,) int64 1-based window start
    strand: np.ndarray         # (N,) uint8
    col_pos: np.ndarray        # (N,) int64 absolute base position in `genome`
    genome: np.ndarray         # packed words of all records
    rec_word_off: np.ndarray
    rec_nbases: np.ndarray
    batch_size: int = 8192
    scales: object = None      # (N,) float32 column scales (scaled form only)
    rows: object = None        # row-layout .bin: Julia (N, rdim) fp16/fp32 as an (rdim, N) array
    _heads: list = field(default=None, repr=False)

    @property
    def N(self) -> int:
        return int(self.col_rec.size)

    @property
    def rdim(self) -> int:
        return 2 * self.m * 4 ** self.c

    @property
    def encoder(self) -> RopeEncoder:
        return RopeEncoder(k=self.k, s=self.s, m=self.m, c=self.c)

    @property
    def heads(self) -> list:
        """Per-column verbatim record header (the reference's `heads` field)."""
        if self._heads is None:
            self._heads = [self.rec_heads[i] for i in self.col_rec]
        return self._heads

    @property
    def scaled(self) -> bool:
        return self.format == SCALED_FORMAT

    def save(self, path) -> None:
        save_index(self, path)


def build_index(re: RopeEncoder, source, kstep: int | None = None, batch_size: int = 8192,
                normalize: int = 0, scaled: bool = False, device=None, stream=None,
                pack: RefPack | None = None) -> Index:
    """build_index_matrix + _index_data_nt (build.jl:694-768), on the GPU.

    source: a FASTA path or bytes (ignored when `pack` is given).  The
    e4m3 columns stay on `device` (the resident database B).
    """
    if kstep is None:
        kstep = max(re.k // 10, 1)
    if kstep < 1 or batch_size < 1:
        raise ValueError("kstep and batch_size must be >= 1")
    _lib.require_device()
    if pack is None:
        pack = pack_reference(source)
        src_name = "<bytes>" if isinstance(source, (bytes, bytearray)) else os.path.abspath(source)
    else:
        src_name = str(source)
    pos, rec, st = window_positions(pack, re.k, kstep)
    nwin = pos.size
    col_win, strand = batch_column_order(nwin, batch_size)
    N = 2 * nwin
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    B = torch.empty((N, re.rdim), dtype=torch.uint8, device=dev)
    norms = torch.empty((N, re.m), dtype=torch.float32, device=dev)
    scales = torch.empty((N,), dtype=torch.float32, device=dev) if scaled else None
    if nwin:
        g = torch.from_numpy(pack.words.view(np.int32)).to(dev)
        p = torch.from_numpy(pos).to(dev)
        kind = _lib.OUT_E4M3_SCALED if scaled else _lib.OUT_E4M3
        check(lib().r2m_encode_ref_windows(ptr(B), kind, ptr(norms), ptr(scales), ptr(g), ptr(p), nwin,
                                           batch_size, re.k, re.s, re.m, re.c, normalize,
                                           stream_handle(stream)))
        torch.cuda.current_stream(dev).synchronize() if stream is None else stream.synchronize()
        del g, p
    return Index(format=SCALED_FORMAT if scaled else FP8_FORMAT, source=src_name, k=re.k, kstep=kstep,
                 s=re.s, m=re.m, c=re.c, normalize=normalize, n_frag=nwin, embeds8=B,
                 norms=norms.cpu().numpy(), rec_heads=list(pack.heads),
                 col_rec=rec[col_win] if nwin else np.zeros(0, np.int32),
                 starts=st[col_win] if nwin else np.zeros(0, np.int64), strand=strand,
                 col_pos=pos[col_win] if nwin else np.zeros(0, np.int64), genome=pack.words,
                 rec_word_off=pack.word_off, rec_nbases=pack.nbases, batch_size=batch_size,
                 scales=scales)


def build_index_packed(re: RopeEncoder, words, rec_heads, rec_word_off, rec_nbases, kstep: int,
                       batch_size: int = 8192, normalize: int = 0, scaled: bool = False,
                       stream=None, source: str = "packed") -> Index:
    """build_index over a genome that is already packed on the device
    (int32/uint32 words, records on word boundaries with guard words)."""
    _lib.require_device()
    pack = RefPack(list(rec_heads), np.asarray(rec_word_off, np.int64), np.asarray(rec_nbases, np.int64),
                   np.zeros(1, np.uint32))
    pos, rec, st = window_positions(pack, re.k, kstep)
    nwin = pos.size
    col_win, strand = batch_column_order(nwin, batch_size)
    dev = words.device
    N = 2 * nwin
    B = torch.empty((N, re.rdim), dtype=torch.uint8, device=dev)
    norms = torch.empty((N, re.m), dtype=torch.float32, device=dev)
    scales = torch.empty((N,), dtype=torch.float32, device=dev) if scaled else None
    if nwin:
        p = torch.from_numpy(pos).to(dev)
        kind = _lib.OUT_E4M3_SCALED if scaled else _lib.OUT_E4M3
        check(lib().r2m_encode_ref_windows(ptr(B), kind, ptr(norms), ptr(scales), ptr(words), ptr(p), nwin,
                                           batch_size, re.k, re.s, re.m, re.c, normalize,
                                           stream_handle(stream)))
        torch.cuda.synchronize(dev)
    return Index(format=SCALED_FORMAT if scaled else FP8_FORMAT, source=source, k=re.k, kstep=kstep,
                 s=re.s, m=re.m, c=re.c, normalize=normalize, n_frag=nwin, embeds8=B,
                 norms=norms.cpu().numpy(), rec_heads=list(rec_heads),
                 col_rec=rec[col_win], starts=st[col_win], strand=strand, col_pos=pos[col_win],
                 genome=np.zeros(1, np.uint32), rec_word_off=pack.word_off, rec_nbases=pack.nbases,
                 batch_size=batch_size, scales=scales)


# ------------------------------------------------------------------ file I/O

_ARRAYS = ("embeds8", "norms", "col_rec", "starts", "strand", "col_pos", "genome", "rec_word_off",
           "rec_nbases", "scales")


def _host(a):
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def save_index(idx: Index, path, container: bool | None = None) -> None:
    """run_save (build.jl:781-795): the reference's Julia-serialized
    NamedTuple, or (container=True, or a path ending in .r2mi) the flat
    container that also keeps the packed genome (see module doc)."""
    if container is None:
        container = os.fspath(path).endswith(".r2mi")
    if container:
        _save_container(idx, path)
    else:
        _save_bin(idx, path)


def _save_bin(idx: Index, path) -> None:
    """_index_data_nt(...; fp8 = true) + save (build.jl:755-768,
    dna.jl:23-27): the 15 fields in the reference's order.  The scaled form
    (a format of this library) adds its column scales as a 16th field."""
    from . import jlbin
    emb = _host(idx.embeds8)
    fields = [("format", idx.format), ("source", idx.source), ("k", int(idx.k)), ("kstep", int(idx.kstep)),
              ("s", int(idx.s)), ("m", int(idx.m)), ("c", int(idx.c)), ("normalize", int(idx.normalize)),
              ("fp8", True), ("n_frag", int(idx.n_frag)), ("embeds8", jlbin.E4M3(emb)),
              ("norms", np.ascontiguousarray(_host(idx.norms), dtype=np.float32)),
              ("heads", jlbin.StrVec(list(idx.rec_heads), np.asarray(idx.col_rec, np.int32))),
              ("starts", np.ascontiguousarray(idx.starts, dtype=np.int64)),
              ("strand", np.ascontiguousarray(idx.strand, dtype=np.uint8))]
    if idx.scaled:
        fields.append(("scales", np.ascontiguousarray(_host(idx.scales), dtype=np.float32)))
    jlbin.write_bin(path, fields)


def _save_container(idx: Index, path) -> None:
    meta = dict(format=idx.format, source=idx.source, k=idx.k, kstep=idx.kstep, s=idx.s, m=idx.m,
                c=idx.c, normalize=idx.normalize, fp8=True, n_frag=idx.n_frag,
                batch_size=idx.batch_size, rec_heads=idx.rec_heads, arrays={})
    arrays = {}
    for name in _ARRAYS:
        if getattr(idx, name) is None:
            if name == "scales":
                continue
            raise ValueError(f"the container needs {name}; an index read from a reference .bin has no "
                             "packed genome (build it from its FASTA)")
        a = _host(getattr(idx, name))
        if a is not None:
            arrays[name] = np.ascontiguousarray(a)
    off = 0
    for name, a in arrays.items():
        meta["arrays"][name] = dict(dtype=a.dtype.str, shape=list(a.shape), offset=off)
        off += (a.nbytes + 63) // 64 * 64
    hdr = json.dumps(meta).encode()
    base = (len(_MAGIC) + 8 + len(hdr) + 63) // 64 * 64
    with open(path, "wb") as f:
        f.write(_MAGIC)
        f.write(np.uint64(len(hdr)).tobytes())
        f.write(hdr)
        f.write(b"\0" * (base - len(_MAGIC) - 8 - len(hdr)))
        pos = 0
        for name, a in arrays.items():
            o = meta["arrays"][name]["offset"]
            if o > pos:
                f.write(b"\0" * (o - pos))
                pos = o
            f.write(a.tobytes())
            pos += a.nbytes


def load_index(path, device=None, mmap: bool = True) -> Index:
    """load_index (load.jl:49-73): structural checks, normalize == 0 required.

    Reads the reference's .bin (Julia-serialized NamedTuple, fp8 column or
    fp16/fp32 row layout) or the flat container.  embeds8 stays on the host
    (memory-mapped) unless `device` is given, in which case it is uploaded
    once (index_database, load.jl:156-161).
    """
    path = os.fspath(path)
    if not os.path.isfile(path):
        raise FileNotFoundError(f"index .bin not found: {path}")
    with open(path, "rb") as f:
        head = f.read(8)
    from . import jlbin
    if head[:3] == jlbin.JULIA_MAGIC:
        return _load_bin(path, device, mmap)
    if head != _MAGIC:
        raise ValueError(f"not an {ROW_FORMAT}/{FP8_FORMAT} index: {path}")
    with open(path, "rb") as f:
        f.read(8)
        hl = int(np.frombuffer(f.read(8), np.uint64)[0])
        meta = json.loads(f.read(hl))
    base = (len(_MAGIC) + 8 + hl + 63) // 64 * 64
    if meta.get("format") not in (FP8_FORMAT, SCALED_FORMAT):
        raise ValueError(f"not an {FP8_FORMAT} index: {path}")
    if meta["normalize"] != 0:
        raise ValueError(f"mapping assumes a normalize = 0 index (got {meta['normalize']})")
    arrs = {}
    for name, d in meta["arrays"].items():
        shape = tuple(d["shape"])
        if mmap:
            arrs[name] = np.memmap(path, dtype=np.dtype(d["dtype"]), mode="r", offset=base + d["offset"],
                                   shape=shape) if int(np.prod(shape)) else np.zeros(shape, np.dtype(d["dtype"]))
        else:
            with open(path, "rb") as f:
                f.seek(base + d["offset"])
                arrs[name] = np.frombuffer(f.read(int(np.prod(shape)) * np.dtype(d["dtype"]).itemsize),
                                           np.dtype(d["dtype"])).reshape(shape)
    rdim = 2 * meta["m"] * 4 ** meta["c"]
    N = 2 * meta["n_frag"]
    if tuple(arrs["embeds8"].shape) != (N, rdim):
        raise ValueError("embeds8 shape mismatch")
    for nm in ("col_rec", "starts", "strand"):
        if arrs[nm].shape[0] != N:
            raise ValueError("meta length mismatch")
    emb = arrs["embeds8"]
    scales = arrs.get("scales")
    if device is not None:
        emb = torch.from_numpy(np.ascontiguousarray(emb)).to(device)
        if scales is not None:
            scales = torch.from_numpy(np.ascontiguousarray(scales)).to(device)
    return Index(format=meta["format"], source=meta["source"], k=meta["k"], kstep=meta["kstep"],
                 s=meta["s"], m=meta["m"], c=meta["c"], normalize=meta["normalize"],
                 n_frag=meta["n_frag"], embeds8=emb, norms=arrs["norms"], rec_heads=meta["rec_heads"],
                 col_rec=arrs["col_rec"], starts=arrs["starts"], strand=arrs["strand"],
                 col_pos=arrs["col_pos"], genome=arrs["genome"], rec_word_off=arrs["rec_word_off"],
                 rec_nbases=arrs["rec_nbases"], batch_size=meta.get("batch_size", 8192),
                 scales=scales)


def _load_bin(path, device, mmap: bool) -> Index:
    """The reference's .bin: the checks of load_index (load.jl:49-73) on the
    NamedTuple that _index_data_nt writes (build.jl:755-772)."""
    from . import jlbin
    d, _ = jlbin.read_bin(path, mmap=mmap)
    fmt = d.get("format")
    fp8 = fmt in (FP8_FORMAT, LEGACY_FP8_FORMAT, SCALED_FORMAT)
    if not (fp8 or fmt in (ROW_FORMAT, LEGACY_ROW_FORMAT)):
        raise ValueError(f"not an {ROW_FORMAT}/{FP8_FORMAT} index: {path}")
    for key in ("k", "kstep", "s", "m", "c", "normalize", "n_frag", "norms", "heads", "starts", "strand"):
        if key not in d:
            raise ValueError(f"index .bin lacks the field {key}: {path}")
    if d["normalize"] != 0:
        raise ValueError(f"mapping assumes a normalize = 0 index (got {d['normalize']}): "
                         "unit-energy rows are what makes B's columns normalized")
    rdim = 2 * d["m"] * 4 ** d["c"]
    N = 2 * d["n_frag"]
    rows = None
    if fp8:
        emb = d.get("embeds8")
        if not isinstance(emb, jlbin.E4M3Array):
            raise ValueError("embeds8 eltype mismatch")
        if tuple(emb.shape) != (N, rdim):  # Julia (rdim, N)
            raise ValueError("embeds8 shape mismatch")
        emb = emb.view(np.ndarray)
    else:
        rows = d.get("embeds")
        want = np.float16 if d.get("fp16", False) else np.float32
        if not isinstance(rows, np.ndarray) or rows.dtype != want:
            raise ValueError("embeds eltype mismatch")
        if tuple(rows.shape) != (rdim, N):  # Julia (N, rdim), column-major
            raise ValueError("embeds shape mismatch")
        emb = None
    heads, starts, strand, norms = d["heads"], d["starts"], d["strand"], d["norms"]
    if not (isinstance(heads, jlbin.StrVec) and len(heads) == starts.shape[0] == strand.shape[0] == N):
        raise ValueError("meta length mismatch")
    if tuple(norms.shape) != (N, d["m"]):
        raise ValueError("norms shape mismatch")
    scales = d.get("scales") if fmt == SCALED_FORMAT else None
    idx = Index(format=SCALED_FORMAT if fmt == SCALED_FORMAT else FP8_FORMAT, source=d.get("source", ""),
                k=d["k"], kstep=d["kstep"], s=d["s"], m=d["m"], c=d["c"], normalize=0, n_frag=d["n_frag"],
                embeds8=emb, norms=norms, rec_heads=list(heads.uniq), col_rec=heads.idx,
                starts=starts, strand=strand, col_pos=None, genome=None,
                rec_word_off=np.zeros(0, np.int64), rec_nbases=np.zeros(0, np.int64), scales=scales)
    idx.rows = rows
    if device is not None:
        idx.embeds8 = index_database(idx, device)
        if scales is not None:
            idx.scales = torch.from_numpy(np.ascontiguousarray(scales)).to(device)
    return idx


def attach_genome(idx: Index, fasta=None) -> Index:
    """Give an index read from a reference .bin (which stores no packed
    genome) the packed records and per-column genome positions that FP32
    rescoring re-encodes windows from: the source FASTA (`fasta`, default
    the index's `source` field) is packed again and each column's record is
    found by its verbatim header."""
    src = fasta if fasta is not None else idx.source
    if not src or not os.path.isfile(os.fspath(src)):
        raise ValueError(f"the index's source FASTA is not available ({src!r}); pass fasta=")
    pack = pack_reference(src)
    where = {}
    for r, h in enumerate(pack.heads):
        if h in where:
            raise ValueError(f"duplicate record header {h!r} in {src}: columns cannot be placed")
        where[h] = r
    try:
        rec_of = np.array([where[h] for h in idx.rec_heads], np.int64)
    except KeyError as e:
        raise ValueError(f"record {e.args[0]!r} of the index is not in {src}") from None
    col_rec = np.asarray(idx.col_rec, np.int64)
    recs = rec_of[col_rec]
    starts0 = np.asarray(idx.starts, np.int64) - 1
    if np.any(starts0 < 0) or np.any(starts0 + idx.k > pack.nbases[recs]):
        raise ValueError(f"index windows do not fit the records of {src}")
    idx.col_pos = 16 * pack.word_off[recs] + starts0
    idx.genome, idx.rec_word_off, idx.rec_nbases = pack.words, pack.word_off, pack.nbases
    return idx


def index_to_f8(rows, device=None, block: int = 1 << 16, stream=None) -> torch.Tensor:
    """index_to_f8 (load.jl:75-97): the row-layout index (Julia (N, rdim)
    fp16/fp32, here its column-major bytes as an (rdim, N) array) -> the
    e4m3 database B, block by block: H2D, transpose, quantise (the library's
    cvt.rn.satfinite conversion, fp16 -> fp32 -> e4m3 like the reference)."""
    _lib.require_device()
    rdim, N = rows.shape
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    B = torch.empty((N, rdim), dtype=torch.uint8, device=dev)
    conv = lib().r2m_f16_to_e4m3 if rows.dtype == np.float16 else lib().r2m_f32_to_e4m3
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    with torch.cuda.stream(st):
        for j0 in range(0, N, block):
            j1 = min(N, j0 + block)
            blk = torch.from_numpy(np.ascontiguousarray(rows[:, j0:j1])).to(dev, non_blocking=False)
            t = blk.t().contiguous()
            check(conv(ptr(B[j0:j1]), ptr(t), t.numel(), st.cuda_stream))
    st.synchronize()
    return B


def index_database(idx: Index, device=None) -> torch.Tensor:
    """index_database (load.jl:156-161): the resident e4m3 database B on the
    GPU -- one H2D for the fp8 layout, index_to_f8 for the row layout."""
    if isinstance(idx.embeds8, torch.Tensor) and idx.embeds8.is_cuda:
        return idx.embeds8
    dev = device if device is not None else "cuda"
    if idx.embeds8 is None:
        if getattr(idx, "rows", None) is None:
            raise ValueError("index holds no embeddings")
        return index_to_f8(idx.rows, dev)
    return torch.from_numpy(np.ascontiguousarray(idx.embeds8)).to(dev)
