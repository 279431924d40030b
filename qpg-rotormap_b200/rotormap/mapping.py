"""Mapping entry points: the tools/map.jl table writer and map_and_count.

Mirrors RotorMap/tools/map.jl:100-184 (run_map), RotorMap/search/
engine_fp8.jl:654-733 (map_and_count) and RotorMap/reads/provenance.jl:46-78
(parse_read_head).
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from .engine import TopKEngine, rope_topk_stream
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


def julia_repr_f32(x: float) -> str:
    """Julia's `string(::Float32)`: shortest round-trip digits, decimal form
    for 1e-4 <= |x| < 1e6, else `d.ddde±x` (the score field of map.jl:148)."""
    x = np.float32(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "Inf" if x > 0 else "-Inf"
    if x == 0:
        return "-0.0" if math.copysign(1.0, float(x)) < 0 else "0.0"
    r = repr(x)  # numpy: shortest round-trip for float32, e.g. '0.9873047' / '1e-05'
    r = r.replace("np.float32(", "").rstrip(")")
    sign = "-" if r.startswith("-") else ""
    r = r.lstrip("-")
    # split into digits and decimal exponent
    if "e" in r:
        mant, ex = r.split("e")
        ex = int(ex)
    else:
        mant, ex = r, 0
    if "." in mant:
        ip, fp = mant.split(".")
    else:
        ip, fp = mant, ""
    digits = (ip + fp).lstrip("0")
    lead_zeros = len(ip + fp) - len((ip + fp).lstrip("0"))
    # decimal exponent of the first significant digit
    e10 = len(ip) - 1 + ex - lead_zeros
    digits = digits.rstrip("0") or "0"
    if -5 < e10 < 6:
        if e10 >= 0:
            ip2 = digits[:e10 + 1].ljust(e10 + 1, "0")
            fp2 = digits[e10 + 1:] or "0"
        else:
            ip2 = "0"
            fp2 = "0" * (-e10 - 1) + digits
        return f"{sign}{ip2}.{fp2}"
    fp2 = digits[1:] or "0"
    return f"{sign}{digits[0]}.{fp2}e{e10}"


def write_table(io, vals, locs, heads, idx: Index, recname=None) -> int:
    """Write map.jl's match lines for one batch (map.jl:141-151):
    `<read hdr sans '>'> <+|-> <score> <starts[c]-1> <record first token>`."""
    if recname is None:
        recname = [_no_gt(h.split()[0]) if h.split() else "" for h in idx.rec_heads]
    lines = []
    for r in range(vals.shape[0]):
        hd = _no_gt(heads[r])
        for j in range(vals.shape[1]):
            c = int(locs[r, j]) - 1
            lines.append(f"{hd} {'+' if idx.strand[c] == 0 else '-'} {julia_repr_f32(vals[r, j])} "
                         f"{int(idx.starts[c]) - 1} {recname[idx.col_rec[c]]}\n")
    io.write("".join(lines))
    return len(lines)


def run_map(index, reads, out=None, topk: int = 20, batch_size: int = 8192, verbose: bool = False,
            score: str | None = None) -> int:
    """run_map (map.jl:100-184): INDEX + READS -> the match table at `out`
    (default READS + ".maps").  Returns the number of reads mapped."""
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
    with open(out, "w") as io:
        for bat in rope_topk_stream(idx.encoder, reads, B, k=topk, batch_size=batch_size, score=score,
                                    scaleB=sb):
            write_table(io, bat.vals, bat.locs, bat.heads, idx, recname)
            n += len(bat.heads)
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
