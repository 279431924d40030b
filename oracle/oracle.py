"""CPU oracle for RotorMap's read-mapping hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs may import this module; the product path (qpg-rotormap_b200/) never does.

Pure-Python / numpy restatements (each cites the reference code it follows,
paths relative to the q4bio-qpg/qpg-rotormap tree):
  fasta_reads_ref     RotorMap/fasta/reader.jl:21-28,61-75,120-198,204-311
  forward_pack        RotorMap/common/harness.jl:112-118 (_ref_forward_pack)
  frag_codes          RotorMap/encode/reference.jl:29-35 (_frag_codes)
  revcomp_words_ref   RotorMap/index/build.jl:415-423 (_revcomp_words_ref)
  ref_windows_ref     RotorMap/index/build.jl:291-324 (_each_ref_window!) and
                      RotorMap/common/harness.jl:52-91 (_e2h_ref_table)
  parse_read_head     RotorMap/reads/provenance.jl:46-78
  map_and_count_ref   RotorMap/search/engine_fp8.jl:654-733 (scoring loop)
  seg_topk_merge_ref  RotorMap/gemm/topk_kernels.jl:213-329 (segmented top-k,
                      its reservoir / merge tie rules)
  batch_topk_ref      RotorMap/search/engine_fp8.jl:399-437 (chunk loop)
  julia_repr_f32_ref  Julia's string(::Float32), the score field of
                      RotorMap/tools/map.jl:148
  table_lines_ref     RotorMap/tools/map.jl:141-151 (match table lines)
C restatements (oracle/rotormap_oracle.c, built by oracle/Makefile):
  rope_f64 / rope_f32 / f32_to_e4m3 / f32_to_f16 / topk_e4m3 / scores_e4m3.

Parity status: pinned against the reference's own outputs.  The reference
(Julia) cannot run here, but it commits three encoder sweep curves
(RotorMap/experiments/out/rope_*_sweep.csv: its fp64 encoder at k = 20,000,
s5 m1 c5, on fixtures drawn from Julia's Xoshiro).  rotormap.jlrandom
reproduces those fixtures draw for draw, and rope_f64 reproduces the
curves' float64 inner products to within 1e-12 (observed <= 7e-16;
tests/golden/rope_sweeps.json, tests/test_cpu_oracle.py).  The reference's
known-answer properties and hand-derived vectors (tests/golden/) cover the
rest (s > c scramble, m > 1, quantisation, top-k).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

_LUT = np.full(256, 2, dtype=np.uint8)
for _ch, _code in (("A", 0), ("C", 1), ("G", 2), ("T", 3), ("a", 0), ("c", 1), ("g", 2), ("t", 3)):
    _LUT[ord(_ch)] = _code


def build() -> Path:
    """Compile oracle/_build/liboracle.so from rotormap_oracle.c (gcc)."""
    src = HERE / "rotormap_oracle.c"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.c_void_p
        i64 = ctypes.c_int64
        ci = ctypes.c_int
        L.orc_rope_batch_f64.argtypes = [P, i64, ci, ci, ci, ci, ci, P, P, ci]
        L.orc_rope_batch_f32.argtypes = [P, i64, ci, ci, ci, ci, ci, P, P, ci]
        L.orc_f32_to_e4m3_array.argtypes = [P, P, i64]
        L.orc_f32_to_f16_array.argtypes = [P, P, i64]
        L.orc_topk_e4m3.argtypes = [P, P, i64, i64, ci, ci, ci, P, P, P, P, ci]
        L.orc_scores_e4m3.argtypes = [P, P, i64, ci, ci, P, P]
        L.orc_e4m3_to_f32.argtypes = [ctypes.c_uint8]
        L.orc_e4m3_to_f32.restype = ctypes.c_float
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _threads(n):
    return n if n else (os.cpu_count() or 1)


# ---------------------------------------------------------------- encoders


def rope_f64(words: np.ndarray, k: int, s: int, m: int, c: int, normalize: int = 0,
             nthreads: int = 0):
    """fp64 golden encoder over (n, W) forward words -> (out (n, rdim), norms (n, m))."""
    words = np.ascontiguousarray(words, dtype=np.uint32)
    n = words.shape[0]
    rdim = 2 * m * 4 ** c
    out = np.zeros((n, rdim), np.float64)
    norms = np.zeros((n, m), np.float64)
    rc = lib().orc_rope_batch_f64(_p(words), n, k, s, m, c, normalize, _p(out), _p(norms), _threads(nthreads))
    assert rc == 0
    return out, norms


def rope_f32(words: np.ndarray, k: int, s: int, m: int, c: int, normalize: int = 0,
             nthreads: int = 0):
    """fp32 kernel-arithmetic encoder -> (out (n, rdim) f32, norms (n, m) f32)."""
    words = np.ascontiguousarray(words, dtype=np.uint32)
    n = words.shape[0]
    rdim = 2 * m * 4 ** c
    out = np.zeros((n, rdim), np.float32)
    norms = np.zeros((n, m), np.float32)
    rc = lib().orc_rope_batch_f32(_p(words), n, k, s, m, c, normalize, _p(out), _p(norms), _threads(nthreads))
    assert rc == 0
    return out, norms


def f32_to_e4m3(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.shape, np.uint8)
    lib().orc_f32_to_e4m3_array(_p(x), _p(out), x.size)
    return out


def f32_to_f16_bits(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.shape, np.uint16)
    lib().orc_f32_to_f16_array(_p(x), _p(out), x.size)
    return out


def e4m3_table() -> np.ndarray:
    L = lib()
    return np.array([L.orc_e4m3_to_f32(i) for i in range(256)], dtype=np.float32)


def quantize_parity(x: np.ndarray) -> np.ndarray:
    """The reference's e4m3 of an encoder output: e4m3(fp32(fp16(x)))."""
    h = f32_to_f16_bits(np.asarray(x, np.float32)).view(np.float16).astype(np.float32)
    return f32_to_e4m3(h)


def quantize_scaled(x: np.ndarray):
    """Per-row scaled e4m3: q = e4m3(x * 448/amax), scale = amax/448."""
    x = np.asarray(x, np.float32)
    amax = np.abs(x).max(axis=1)
    mul = np.where(amax > 0, np.float32(448.0) / np.where(amax > 0, amax, 1), 1).astype(np.float32)
    q = f32_to_e4m3((x * mul[:, None]).astype(np.float32))
    scale = np.where(amax > 0, amax / np.float32(448.0), 0).astype(np.float32)
    return q, scale


# ---------------------------------------------------------------- search


def topk_e4m3(A: np.ndarray, B: np.ndarray, k: int, mode: int = 0, scaleA=None, scaleB=None,
              nthreads: int = 0):
    """Brute-force top-k of e4m3 reads A (nb, rdim) vs index columns B (N, rdim).

    mode 0: fp16-rounded fp32 scores, 1: fp32, 2: fp32 * scaleA * scaleB.
    Returns vals (nb, k) f32 descending (ties by column asc), locs (nb, k) 1-based.
    """
    A = np.ascontiguousarray(A, dtype=np.uint8)
    B = np.ascontiguousarray(B, dtype=np.uint8)
    nb, rdim = A.shape
    N = B.shape[0]
    vals = np.empty((nb, k), np.float32)
    locs = np.empty((nb, k), np.int32)
    sa = np.ascontiguousarray(scaleA if scaleA is not None else np.ones(nb), dtype=np.float32)
    sb = np.ascontiguousarray(scaleB if scaleB is not None else np.ones(N), dtype=np.float32)
    lib().orc_topk_e4m3(_p(A), _p(B), nb, N, rdim, k, mode, _p(sa), _p(sb), _p(vals), _p(locs),
                        _threads(nthreads))
    return vals, locs


def scores_e4m3(a8: np.ndarray, B: np.ndarray, mode: int = 0, scaleB=None) -> np.ndarray:
    a8 = np.ascontiguousarray(a8, dtype=np.uint8)
    B = np.ascontiguousarray(B, dtype=np.uint8)
    N, rdim = B.shape
    sb = np.ascontiguousarray(scaleB if scaleB is not None else np.ones(N), dtype=np.float32)
    out = np.empty(N, np.float32)
    lib().orc_scores_e4m3(_p(a8), _p(B), N, rdim, mode, _p(sb), _p(out))
    return out


# ---------------------------------------------------------------- packing


def forward_pack(codes: np.ndarray, L: int) -> np.ndarray:
    """Base j -> word j>>4, bits 2*(j&15); zero tail (harness.jl:112-118)."""
    words = np.zeros((L + 15) // 16, np.uint32)
    for j in range(L):
        words[j >> 4] |= np.uint32(int(codes[j]) << (2 * (j & 15)))
    return words


def frag_codes(words: np.ndarray, k: int) -> np.ndarray:
    """reference.jl:29-35."""
    return np.array([(int(words[j >> 4]) >> (2 * (j & 15))) & 3 for j in range(k)], np.uint8)


def revcomp_words_ref(words: np.ndarray, k: int) -> np.ndarray:
    """Codes-based reverse complement (build.jl:415-423)."""
    codes = frag_codes(words, k)
    rc = np.array([3 - codes[k - 1 - j] for j in range(k)], np.uint8)
    return forward_pack(rc, k)


def _is_rec_start(raw: bytes, t: int) -> bool:
    return raw[t] == 0x3E and (t == 0 or raw[t - 1] in (0x0A, 0x0D))


def _next_rec(raw: bytes, frm: int) -> int:
    """First line-start '>' at index >= frm, else len(raw) (reader.jl:61-75)."""
    n = len(raw)
    p = frm
    while p < n:
        t = raw.find(b">", p)
        if t < 0:
            return n
        if _is_rec_start(raw, t):
            return t
        p = t + 1
    return n


def fasta_reads_ref(raw: bytes, k: int):
    """Single-part semantics of fasta_reads: [(header, words)] in file order."""
    out = []
    n = len(raw)
    s = _next_rec(raw, 0)
    while s < n:
        e = _next_rec(raw, s + 1)
        h = s
        while h < e and raw[h] != 0x0A:
            h += 1
        if h == e:
            break  # header line not closed: the part ends inside it
        hend = h
        if hend > s and raw[hend - 1] == 0x0D:
            hend -= 1
        codes = []
        for b in raw[h + 1:e]:
            if len(codes) >= k:
                break
            if b in (0x0A, 0x0D):
                continue
            codes.append(int(_LUT[b]))
        if len(codes) >= k:
            out.append((raw[s:hend].decode("latin-1"), forward_pack(np.array(codes, np.uint8), k)))
        s = e
    return out


def ref_table(raw: bytes):
    """Records -> (headers, codes arrays) with _LUT3 codes (harness.jl:52-91)."""
    heads, seqs = [], []
    n = len(raw)
    s = _next_rec(raw, 0)
    while s < n:
        h = s
        while h < n and raw[h] != 0x0A:
            h += 1
        hend = h
        if hend > s and raw[hend - 1] == 0x0D:
            hend -= 1
        e = _next_rec(raw, s + 1)
        body = np.frombuffer(raw[h + 1:e] if h + 1 <= e else b"", dtype=np.uint8)
        body = body[(body != 0x0A) & (body != 0x0D)]
        heads.append(raw[s:hend].decode("latin-1"))
        seqs.append(_LUT[body])
        s = e
    return heads, seqs


def ref_windows_ref(raw: bytes, k: int, kstep: int):
    """Every k-window (offsets 0, kstep, ... fully inside) of every record:
    [(header, start_1based, forward words)] in file order (build.jl:291-324)."""
    out = []
    heads, seqs = ref_table(raw)
    for hd, codes in zip(heads, seqs):
        if len(codes) < k:
            continue
        nwin = (len(codes) - k) // kstep + 1
        for wi in range(nwin):
            off = wi * kstep
            out.append((hd, off + 1, forward_pack(codes[off:off + k], k)))
    return out


# ---------------------------------------------------------------- scoring


def parse_read_head(h: str):
    """provenance.jl:46-78 -> dict(id, start (1-based), len or None, src) or None."""
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
    rev = f[2].split("#")[0]
    if rev not in ("true", "false"):
        return None
    return dict(id=h, start=start + 1, len=None, src=f[0][1:])


def map_and_count_ref(heads, locs, db_heads, db_starts, dbk: int, ktop: int):
    """The scoring loop of map_and_count (engine_fp8.jl:668-727) on given
    top-k locations: returns (total, correct, rank_hist, inter_sum, inter_cnt)."""
    rec_id, rec_id_acc = {}, {}
    rec_of_col = []
    for h in db_heads:
        i = rec_id.get(h)
        if i is None:
            i = len(rec_id) + 1
            rec_id[h] = i
            rec_id_acc[h.split()[0][1:]] = i
        rec_of_col.append(i)
    total = correct = inter_sum = inter_cnt = 0
    hist = [0] * ktop
    for r, hd in enumerate(heads):
        h = parse_read_head(hd)
        if h is None:
            raise ValueError(f"unreadable provenance header: {hd}")
        rid = rec_id_acc.get(h["src"], 0)
        hit = ilen = 0
        for j in range(ktop):
            c = int(locs[r][j]) - 1
            ds = db_starts[c]
            if rec_of_col[c] == rid and h["start"] <= ds + dbk - 1 and ds <= h["start"] + dbk - 1:
                if hit == 0:
                    hit = j + 1
                il = min(h["start"] + dbk - 1, ds + dbk - 1) - max(h["start"], ds) + 1
                ilen = max(ilen, il)
        total += 1
        if hit:
            correct += 1
            hist[hit - 1] += 1
            if ilen > 0:
                inter_sum += ilen
                inter_cnt += 1
    return total, correct, hist, inter_sum, inter_cnt


def seg_topk_merge_ref(C: np.ndarray, offset: int, dv: np.ndarray, dl: np.ndarray, K: int = 20, PS: int = 8):
    """One chunk of seg_rowtopk_merge_kernel! (RotorMap/gemm/topk_kernels.jl:213-329)
    in plain Python: C (rows, wi) float32 scores of chunk columns offset+1..,
    dv/dl (rows, K) the running lists (updated in place; ids 1-based)."""
    rows, wi = C.shape
    segw = -(-wi // PS)
    for r in range(rows):
        lists = []
        for s in range(PS):
            lo = s * segw
            cnt = max(0, min(wi, (s + 1) * segw) - lo)
            lk = [-np.inf] * K
            li = [0] * K
            thr, mp = -np.inf, 0
            for c in range(cnt):
                v = float(C[r, lo + c])
                if v > thr:  # replace the tracked minimum
                    lk[mp], li[mp] = v, c + 1
                    mp = min(range(K), key=lambda j: (lk[j], j))  # first minimum
                    thr = lk[mp]
            for i in range(1, K):  # stable insertion sort, descending
                v, d, j = lk[i], li[i], i
                while j > 0 and lk[j - 1] < v:
                    lk[j], li[j] = lk[j - 1], li[j - 1]
                    j -= 1
                lk[j], li[j] = v, d
            lists.append((lk, li))
        run_v, run_l = list(dv[r]), list(dl[r])
        heads = [0] * PS
        pa = 0
        for j in range(K):
            va = run_v[pa] if pa < K else -np.inf
            bv, bs, bli = -np.inf, -1, 0
            for s in range(PS):
                h = heads[s]
                if h < K and bv < lists[s][0][h]:  # ties keep the lowest segment
                    bv, bs, bli = lists[s][0][h], s, lists[s][1][h]
            if va >= bv:
                dv[r, j] = va
                dl[r, j] = run_l[pa] if pa < K else 0
                pa += 1
            else:
                dv[r, j] = bv
                dl[r, j] = 0 if bli == 0 else offset + bs * segw + bli
                heads[bs] += 1
    return dv, dl


def batch_topk_ref(scores: np.ndarray, w: int, K: int = 20, PS: int = 8):
    """batch_gemm_topk!'s chunk loop (RotorMap/search/engine_fp8.jl:399-437)
    over a full (rows, N) score matrix."""
    rows, N = scores.shape
    dv = np.full((rows, K), -np.inf, np.float32)
    dl = np.zeros((rows, K), np.int32)
    for lo in range(0, N, w):
        seg_topk_merge_ref(scores[:, lo:lo + w], lo, dv, dl, K, PS)
    return dv, dl


# ---------------------------------------------------------------- match table


def julia_repr_f32_ref(x: float) -> str:
    """Julia's `string(::Float32)` (the score field of RotorMap/tools/map.jl:148):
    shortest round-trip digits (numpy's float32 repr), decimal form when the
    first significant digit's decimal exponent e has -5 < e < 6, else
    `d.ddde±x`; NaN, Inf, -Inf, 0.0, -0.0 literal."""
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


def table_lines_ref(vals, locs, heads, strand, starts, col_rec, recname):
    """The match lines of RotorMap/tools/map.jl:141-151 for one batch:
    `<header without '>'> <+|-> <score> <starts[c]-1> <record name>`."""
    lines = []
    for r in range(vals.shape[0]):
        hd = heads[r][1:] if heads[r].startswith(">") else heads[r]
        for j in range(vals.shape[1]):
            c = int(locs[r, j]) - 1
            lines.append(f"{hd} {'+' if strand[c] == 0 else '-'} {julia_repr_f32_ref(vals[r, j])} "
                         f"{int(starts[c]) - 1} {recname[col_rec[c]]}\n")
    return "".join(lines)
