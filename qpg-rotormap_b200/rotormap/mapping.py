"""Mapping entry points: the tools/map.jl table writer and map_and_count.

Mirrors RotorMap/tools/map.jl:100-184 (run_map), RotorMap/search/
engine_fp8.jl:654-733 (map_and_count) and RotorMap/reads/provenance.jl:46-78
(parse_read_head).
"""
from __future__ import annotations

import os
import time

import numpy as np
import torch

from .engine import rope_topk_stream
from .index import Index, index_database, load_index


def parse_read_head(h: str):
    """Provenance header -> dict(id, start 1-based, len | None, src) or None.

    Formats (provenance.jl:11-39): ">read_<i> start=<1-based> len=<k> src=<rec>"
    and ">record:start0:true|false[#dup]".
    """
    if not h.startswith(">"):
        return None
    if h.startswith(">read_"):
        sp = h.find(" src=")
        if sp < 0:
            return None
        fields = h[:sp].split()
        if len(fields) < 2:
            return None
        kv = {}
        for f in fields[1:]:
            eq = f.find("=")
            if eq < 0:
                return None
            kv[f[:eq]] = f[eq + 1:]
        if "start" not in kv or "len" not in kv:
            return None
        try:
            start, ln = int(kv["start"]), int(kv["len"])
        except ValueError:
            return None
        return dict(id=fields[0], start=start, len=ln, src=h[sp + 5:])
    f = h.split(":")
    if len(f) != 3:
        return None
    try:
        start = int(f[1])
    except ValueError:
        return None
    if f[2].split("#")[0] not in ("true", "false"):
        return None
    return dict(id=h, start=start + 1, len=None, src=f[0][1:])


def _no_gt(s: str) -> str:
    return s[1:] if s.startswith(">") else s


def write_table(io, vals, locs, heads, idx: Index, recname=None, nthreads: int | None = None) -> int:
    """Write map.jl's match lines for one batch (map.jl:141-151):
    `<read hdr sans '>'> <+|-> <score> <starts[c]-1> <record first token>`,
    formatted by the library's native writer (r2m_format_table).  `io` may be
    a binary or a text stream."""
    import ctypes
    import io as _io

    from ._lib import check, lib
    if recname is None:
        recname = [_no_gt(h.split()[0]) if h.split() else "" for h in idx.rec_heads]
    vals = np.ascontiguousarray(vals, np.float32)
    locs = np.ascontiguousarray(locs, np.int32)
    nb, k = vals.shape
    if nb == 0:
        return 0
    from .fasta import HeaderList
    if isinstance(heads, HeaderList):
        hb = heads.blob()
    else:
        hb = ("\n".join(heads) + "\n").encode("latin-1")
    rb = ("\n".join(recname) + "\n").encode("latin-1")
    strand = np.ascontiguousarray(idx.strand, np.uint8)
    starts = np.ascontiguousarray(idx.starts, np.int64)
    col_rec = np.ascontiguousarray(idx.col_rec, np.int32)
    L = lib()
    h = ctypes.c_void_p()
    check(L.r2m_format_table(vals.ctypes.data, locs.ctypes.data, nb, k, hb, len(hb), strand.ctypes.data,
                             starts.ctypes.data, col_rec.ctypes.data, strand.size, rb, len(rb),
                             nthreads or (os.cpu_count() or 1), ctypes.byref(h)))
    try:
        n = ctypes.c_size_t()
        p = L.r2m_text_data(h, ctypes.byref(n))
        if n.value:
            # written straight from the library's buffer (no bytes copy)
            view = memoryview((ctypes.c_char * n.value).from_address(p)).cast("B")
            if isinstance(io, _io.TextIOBase):
                io.write(bytes(view).decode("latin-1"))
            else:
                io.write(view)
            view.release()
    finally:
        L.r2m_text_free(h)
    return nb * k


def julia_repr_f32(x: float) -> str:
    """Julia's `string(::Float32)` (the score field of map.jl:148): shortest
    round-trip digits, decimal form for 1e-4 <= |x| < 1e6, else `d.ddde±x`;
    formatted by the library (r2m_format_f32)."""
    import ctypes

    from ._lib import lib
    buf = ctypes.create_string_buffer(48)
    n = lib().r2m_format_f32(float(x), buf, 48)
    if n < 0:
        raise ValueError("format failed")
    return buf.value.decode()


def run_map(index, reads, out=None, topk: int = 20, batch_size: int = 8192, verbose: bool = False,
            score: str | None = None, reader: str = "auto") -> int:
    """run_map (map.jl:100-184): INDEX + READS -> the match table at `out`
    (default READS + ".maps").  Returns the number of reads mapped.

    The table of batch i is formatted and written by a writer thread (the
    native formatter releases the GIL) while the GPU maps batch i+1."""
    import queue
    import threading

    idx = index if isinstance(index, Index) else load_index(index)
    out = out or (str(reads) + ".maps")
    t0 = time.perf_counter()
    B = index_database(idx)
    sb = None
    if idx.scaled:
        sb = idx.scales if isinstance(idx.scales, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(idx.scales))
        sb = sb.to(B.device)
    score = score or ("scaled" if idx.scaled else "f16")
    recname = [_no_gt(h.split()[0]) if h.split() else "" for h in idx.rec_heads]
    n = 0
    q: queue.Queue = queue.Queue(maxsize=2)
    failure: list = []

    def writer(io):
        while True:
            bat = q.get()
            if bat is None:
                return
            if not failure:
                try:
                    write_table(io, bat.vals, bat.locs, bat.heads, idx, recname)
                except BaseException as e:  # reported by the caller after the join
                    failure.append(e)

    with open(out, "wb") as io:
        th = threading.Thread(target=writer, args=(io,), daemon=True)
        th.start()
        try:
            for bat in rope_topk_stream(idx.encoder, reads, B, k=topk, batch_size=batch_size, score=score,
                                        scaleB=sb, reader=reader):
                if failure:
                    break
                q.put(bat)
                n += len(bat.heads)
        finally:
            q.put(None)
            th.join()
    if failure:
        raise failure[0]
    if verbose:
        t = time.perf_counter() - t0
        print(f"MAPPED {n} reads -> {out} ({n * topk} match lines) in {t:.2f} s")
    return n


def score_provenance(heads, locs, idx: Index, ktop: int):
    """The scoring loop of map_and_count (engine_fp8.jl:668-727)."""
    rec_acc = {}
    for i, h in enumerate(idx.rec_heads):
        toks = h.split()
        rec_acc.setdefault(toks[0][1:] if toks else "", i)
    dbk = idx.k
    total = correct = inter_sum = inter_cnt = 0
    hist = np.zeros(ktop, np.int64)
    for r, hd in enumerate(heads):
        h = parse_read_head(hd)
        if h is None:
            raise ValueError(f"unreadable provenance header: {hd}")
        if h["len"] is not None and h["len"] != dbk:
            raise ValueError(f"read {h['id']}: len = {h['len']} != db window length {dbk}")
        rid = rec_acc.get(h["src"], -1)
        c = locs[r, :ktop].astype(np.int64) - 1
        ds = idx.starts[c]
        ok = (idx.col_rec[c] == rid) & (h["start"] <= ds + dbk - 1) & (ds <= h["start"] + dbk - 1)
        total += 1
        if ok.any():
            j = int(np.argmax(ok))
            correct += 1
            hist[j] += 1
            il = (np.minimum(h["start"] + dbk - 1, ds + dbk - 1) - np.maximum(h["start"], ds) + 1)[ok]
            if il.max() > 0:
                inter_sum += int(il.max())
                inter_cnt += 1
    return total, correct, hist, inter_sum, inter_cnt


def map_and_count(re, reads_file, idx: Index, ktop: int = 20, batch_size: int = 8192,
                  score: str | None = None, normalize: int = 0):
    """map_and_count (engine_fp8.jl:654-733) -> dict(total, correct, rank_hist,
    seconds, inter_sum, inter_cnt, nb)."""
    if re.k != idx.k:
        raise ValueError(f"encoder k = {re.k} != db window length {idx.k}")
    B = index_database(idx)
    sb = None
    if idx.scaled:
        sb = idx.scales if isinstance(idx.scales, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(idx.scales))
        sb = sb.to(B.device)
    score = score or ("scaled" if idx.scaled else "f16")
    tot = cor = isum = icnt = nbat = 0
    hist = np.zeros(ktop, np.int64)
    t0 = time.perf_counter()
    for bat in rope_topk_stream(re, reads_file, B, k=ktop, batch_size=batch_size, score=score, scaleB=sb,
                                normalize=normalize):
        nbat += 1
        t, c, h, s_, n_ = score_provenance(bat.heads, bat.locs, idx, ktop)
        tot += t
        cor += c
        hist += h
        isum += s_
        icnt += n_
    return dict(total=tot, correct=cor, rank_hist=hist, seconds=time.perf_counter() - t0,
                inter_sum=isum, inter_cnt=icnt, nb=nbat)
