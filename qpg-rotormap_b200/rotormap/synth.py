"""Seeded synthetic genomes and reads (stand-ins for the reference's fixture
generators in RotorMap/common/dna.jl and RotorMap/reads/sample.jl).

The reference draws its fixtures from Julia's Xoshiro stream;
rotormap.jlrandom reproduces those draws exactly (generate_reference,
mutate, mutate_shift) for fixtures that must equal the reference's.  The
workload generators here keep the reference's shapes and models at any
size with numpy's PCG64:
  * genome: iid bases with a GC fraction, optional N runs (lengths uniform
    in [run_min, run_max]) covering a given fraction of the bases;
  * `:even` read sampling over each record's N-free windows, midpoints of
    equal strata with largest-remainder allocation (sample.jl:474-610);
  * mutation: iid substitutions at rate `err` (each substituted base takes
    one of the three other bases uniformly), or the reference's `mutate`
    model (ceil(n*err) edits, 1/3 sub / ins / del, length kept).
Headers follow the reference's provenance format
`>read_<i> start=<1-based> len=<k> src=<record name>` (sample.jl:469-470).
"""
from __future__ import annotations

import math

import numpy as np

LETTERS = np.frombuffer(b"ACGT", np.uint8)


def random_genome(lengths, seed: int = 1, gc: float = 0.5, n_frac: float = 0.0,
                  run_min: int = 100, run_max: int = 10_000):
    """Records as (codes uint8 0..3, nmask bool) pairs; N positions carry code 2
    (G, the reference's code for any non-ACGT byte) and nmask True."""
    rng = np.random.default_rng(seed)
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    recs = []
    for L in lengths:
        codes = rng.choice(4, size=int(L), p=p).astype(np.uint8)
        nmask = np.zeros(int(L), bool)
        if n_frac > 0:
            target = int(n_frac * L)
            covered = 0
            while covered < target:
                ln = int(rng.integers(run_min, run_max + 1))
                st = int(rng.integers(0, max(1, L - ln)))
                seg = nmask[st:st + ln]
                covered += int((~seg).sum())
                nmask[st:st + ln] = True
            codes[nmask] = 2
        recs.append((codes, nmask))
    return recs


def genome_fasta(heads, recs, width: int = 70) -> bytes:
    """FASTA text of the records (N runs written as 'N')."""
    out = []
    for h, (codes, nmask) in zip(heads, recs):
        s = LETTERS[codes].copy()
        s[nmask] = ord("N")
        out.append(h.encode() + b"\n")
        b = s.tobytes()
        out.extend(b[i:i + width] + b"\n" for i in range(0, len(b), width))
    return b"".join(out)


def _nfree_window_starts(nmask: np.ndarray, k: int) -> np.ndarray:
    """0-based starts of k-windows free of N (sample.jl `nfree` pool)."""
    L = nmask.size
    if L < k:
        return np.zeros(0, np.int64)
    c = np.concatenate([[0], np.cumsum(nmask.astype(np.int64))])
    bad = c[k:] - c[:-k]
    return np.flatnonzero(bad == 0).astype(np.int64)


def even_alloc(w, n: int):
    """_even_alloc (sample.jl:474-485): largest-remainder allocation."""
    w = np.asarray(w, np.float64)
    quota = n * w / w.sum()
    alloc = np.floor(quota).astype(np.int64)
    fr = quota - alloc
    order = sorted(range(len(w)), key=lambda j: (-fr[j], j))
    for t in range(n - int(alloc.sum())):
        alloc[order[t]] += 1
    return alloc


def substitute(codes: np.ndarray, err: float, rng) -> np.ndarray:
    """iid substitutions: each base is replaced with probability err by one of
    the other three bases."""
    out = codes.copy()
    if err <= 0:
        return out
    hit = rng.random(out.size) < err
    shift = rng.integers(1, 4, size=out.size).astype(np.uint8)
    out[hit] = (out[hit] + shift[hit]) % 4
    return out


def mutate_edits(codes: np.ndarray, err: float, rng) -> np.ndarray:
    """The reference's `mutate` (RotorMap/common/dna.jl:120-183): n_err =
    ceil(n*err) edit operations -- n_ins = n_del = floor(n_err/3)
    insertions and deletions, the other n_sub = n_err - 2*n_ins
    substitutions -- so the length stays exactly n.

    Positions as the reference draws them (1-based, uniform): substitutions
    ceil(n*u), sorted, with replacement, each replacing the original base by
    one of the other three; deletions ceil((n-t)*u) for t = 0.., sorted and
    made strictly increasing; insertions ceil((n-n_del)*u), sorted, of a
    uniform base.  Applied in that order -- substitutions, then deletions,
    then insertions at positions of the shortened sequence (the leaf
    semantics of RotorMap/common/treearrays.jl's subsat!/deleteat!/
    insertat!).  The draws come from `rng` (numpy), not Julia's Xoshiro."""
    codes = np.asarray(codes, np.uint8)
    n = codes.size
    n_err = int(math.ceil(n * err))
    n_ins = n_err // 3
    n_del = n_ins
    n_sub = n_err - n_ins - n_del
    if n_err == 0:
        return codes.copy()
    out = codes.copy()
    inds_s = np.sort(np.maximum(np.ceil(n * rng.random(n_sub)).astype(np.int64), 1))
    out[inds_s - 1] = (codes[inds_s - 1] + rng.integers(1, 4, n_sub)) % 4
    t = np.arange(n_del, dtype=np.int64)
    inds_d = np.sort(np.maximum(np.ceil((n - t) * rng.random(n_del)).astype(np.int64), 1))
    for i in range(1, n_del):
        inds_d[i] = max(inds_d[i], inds_d[i - 1] + 1)
    out = np.delete(out, inds_d - 1)
    inds_i = np.sort(np.maximum(np.ceil((n - n_del) * rng.random(n_ins)).astype(np.int64), 1))
    out = np.insert(out, inds_i - 1, rng.integers(0, 4, n_ins).astype(np.uint8))
    return out.astype(np.uint8)


def sample_reads_even(heads, recs, n: int, k: int, err: float = 0.0, seed: int = 42,
                      model: str = "subs"):
    """`:even` draw over the N-free pool (sample.jl:566-582) -> (reads codes
    list, provenance headers, record index, 1-based starts).

    model "subs": iid substitutions at rate err (numpy draws); "mutate": the
    reference's edit model with numpy draws; "reference": the reference
    sampler's own draws (sample.jl:589-604): `Xoshiro(seed)`, one child
    generator per read seeded by `rand(rng, Int64)`, and `mutate` on that
    child (rotormap.jlrandom) -- the reads `sample_reads(...; draw = :even,
    err, seed)` returns for the same records."""
    pools = [_nfree_window_starts(nm, k) for _, nm in recs]
    w = np.array([p.size for p in pools], np.int64)
    if w.sum() == 0:
        raise ValueError(f"no N-free k = {k} window")
    alloc = even_alloc(w, n)
    rng = np.random.default_rng(seed)
    if model == "reference":
        from . import jlrandom
        jl = jlrandom.Xoshiro(seed)
        children = [jlrandom.Xoshiro(jl.rand_i64()) for _ in range(n)]
    reads, hd, rix, starts = [], [], [], []
    i = 0
    for j, nj in enumerate(alloc):
        Wj = int(w[j])
        for t in range(1, int(nj) + 1):
            rank = 1 + ((2 * t - 1) * Wj) // (2 * nj) if nj <= Wj else ((t - 1) % Wj) + 1
            st0 = int(pools[j][rank - 1])
            codes = recs[j][0][st0:st0 + k]
            if model == "subs":
                codes = substitute(codes, err, rng)
            elif model == "reference":
                codes = jlrandom.mutate(codes, err, children[i])
            else:
                codes = mutate_edits(codes, err, rng)
            i += 1
            name = heads[j].split()[0][1:]
            reads.append(codes)
            hd.append(f">read_{i} start={st0 + 1} len={k} src={name}")
            rix.append(j)
            starts.append(st0 + 1)
    return reads, hd, np.array(rix), np.array(starts)


def reads_fasta(heads, reads) -> bytes:
    return b"".join(h.encode() + b"\n" + LETTERS[r].tobytes() + b"\n" for h, r in zip(heads, reads))


def pack_reads(reads, k: int) -> np.ndarray:
    """Forward 2-bit words (n, cld(k,16)) of equal-length code arrays."""
    n = len(reads)
    W = (k + 15) // 16
    codes = np.zeros((n, W * 16), np.uint32)
    for i, r in enumerate(reads):
        codes[i, :k] = r[:k]
    sh = (2 * np.arange(16, dtype=np.uint32))[None, None, :]
    return np.bitwise_or.reduce(codes.reshape(n, W, 16) << sh, axis=2).astype(np.uint32)


# ------------------------------------------------------------------ on-device generators
# Human-scale genomes (3.1 Gbp) are generated and packed on the GPU: numpy
# would need minutes and ~12 GB of host memory for the same job.


def genome_lengths(total: int, nrec: int, lo: float, hi: float, seed: int):
    """Record lengths uniform on [lo, hi], rescaled to `total` bases."""
    rng = np.random.default_rng(seed)
    raw = rng.uniform(lo, hi, nrec)
    L = np.floor(raw / raw.sum() * total).astype(np.int64)
    L[-1] += total - L.sum()
    return L


def n_runs(length: int, frac: float, run_min: int, run_max: int, rng):
    """Sorted, merged N runs [(start, end)) covering ~frac of a record."""
    runs, covered = [], 0
    target = int(frac * length)
    while covered < target:
        ln = int(rng.integers(run_min, run_max + 1))
        st = int(rng.integers(0, max(1, length - ln)))
        runs.append((st, st + ln))
        covered += ln
    runs.sort()
    merged = []
    for s, e in runs:
        if merged and s <= merged[-1][1]:
            merged[-1] = (merged[-1][0], max(merged[-1][1], e))
        else:
            merged.append((s, e))
    return np.array(merged, np.int64).reshape(-1, 2)


def random_genome_packed(lengths, seed: int = 1, gc: float = 0.5, n_frac: float = 0.0,
                         run_min: int = 100, run_max: int = 10_000, device="cuda"):
    """Records of iid bases (GC fraction `gc`, N runs coded as G like the
    reference LUT) packed on the device: returns (words (int32 tensor, each
    record starting on a word and followed by a zero guard word), word_off,
    nbases, runs per record)."""
    import torch
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    chunks, offs, runs = [], [], []
    cur = 0
    sh = (2 * torch.arange(16, device=device, dtype=torch.int32)).view(1, 16)
    p_a = (1 - gc) / 2
    for L in lengths:
        L = int(L)
        nw = (L + 15) // 16
        u = torch.rand(nw * 16, generator=gen, device=device)
        codes = (u >= p_a).to(torch.int32) + (u >= 0.5).to(torch.int32) + (u >= 0.5 + gc / 2).to(torch.int32)
        codes[L:] = 0
        r = n_runs(L, n_frac, run_min, run_max, rng) if n_frac > 0 else np.zeros((0, 2), np.int64)
        if r.size:
            mark = torch.zeros(nw * 16 + 1, dtype=torch.int32, device=device)
            mark.index_add_(0, torch.from_numpy(r[:, 0]).to(device), torch.ones(len(r), dtype=torch.int32, device=device))
            mark.index_add_(0, torch.from_numpy(r[:, 1]).to(device), -torch.ones(len(r), dtype=torch.int32, device=device))
            nmask = torch.cumsum(mark, 0)[:-1] > 0
            codes[nmask] = 2
            del mark, nmask
        w = (codes.view(nw, 16) << sh).sum(dim=1, dtype=torch.int64).to(torch.int32)  # disjoint bits: sum == or
        chunks += [w, torch.zeros(1, dtype=torch.int32, device=device)]
        offs.append(cur)
        cur += nw + 1
        runs.append(r)
        del u, codes
    return torch.cat(chunks), np.array(offs, np.int64), np.asarray(lengths, np.int64), runs


def sample_positions(nbases, runs, n: int, k: int, seed: int):
    """n uniform read starts (record, 0-based offset) whose k-window avoids N runs."""
    rng = np.random.default_rng(seed)
    nb = np.asarray(nbases, np.int64)
    w = np.maximum(nb - k + 1, 0).astype(np.float64)
    recs, offs = [], []
    while len(recs) < n:
        m = n - len(recs)
        r = rng.choice(len(nb), size=2 * m, p=w / w.sum())
        o = (rng.random(2 * m) * w[r]).astype(np.int64)
        for ri, oi in zip(r, o):
            rr = runs[ri]
            if rr.size:
                j = np.searchsorted(rr[:, 0], oi + k)  # runs starting before the window end
                if j > 0 and rr[j - 1, 1] > oi:
                    continue
            recs.append(int(ri))
            offs.append(int(oi))
            if len(recs) == n:
                break
    return np.array(recs), np.array(offs, np.int64)


def extract_reads_packed(words, word_off, recs, offs, k: int, err, seed: int):
    """Reads cut from the packed device genome at (record, offset), with iid
    substitutions at per-read rates `err`, returned as packed (n, cld(k,16))
    host words."""
    import torch
    dev = words.device
    n = len(recs)
    pos = torch.from_numpy(16 * np.asarray(word_off)[recs] + offs).to(dev)
    j = torch.arange(k, device=dev)
    p = pos[:, None] + j[None, :]
    wv = words[(p >> 4)].to(torch.int64) & 0xFFFFFFFF
    codes = ((wv >> (2 * (p & 15))) & 3).to(torch.int32)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    rate = torch.as_tensor(np.broadcast_to(np.asarray(err, np.float32), (n,)).copy(), device=dev)
    hit = torch.rand((n, k), generator=gen, device=dev) < rate[:, None]
    shift = torch.randint(1, 4, (n, k), generator=gen, device=dev, dtype=torch.int32)
    codes = torch.where(hit, (codes + shift) % 4, codes)
    W = (k + 15) // 16
    pad = torch.zeros((n, W * 16), dtype=torch.int64, device=dev)
    pad[:, :k] = codes
    sh = (2 * torch.arange(16, device=dev, dtype=torch.int64)).view(1, 1, 16)
    packed = (pad.view(n, W, 16) << sh).sum(dim=2)
    return packed.to(torch.int64).cpu().numpy().astype(np.uint32)
