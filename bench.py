"""Benchmark of the read-mapping hot path: fused rope encode -> fp8 GEMM +
per-row top-k on B200.

Workload (the kernel-microbench configuration): Q = 65,536 reads of 150 bp
(uniform positions of the genome, 5% iid substitutions, seeded) encoded at
s=8 m=4 c=4 (rdim 2048) against an index of N = 16,777,216 columns (the
forward and reverse-complement windows, k = 150 and stride 15, of a seeded
125,829,255 bp random genome); e4m3 operands with per-row fp32 scales, fp32
accumulation, top-20 per read.  A step = encode the batch from its packed
words already in HBM + the fused GEMM/top-k + the split merge.  The 34 GB
index is far larger than L2, so no flush is needed between steps.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
  N > 1: launched by torch.distributed.run, one rank per GPU; every rank maps
  its own read batch against its own index replica (weak scaling, no
  collective on the data path).
  --impl reference: times the CPU restatement of the reference path (golden
  fp64 encoder + multithreaded brute-force scoring) on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "qpg-rotormap_b200"))
sys.path.insert(0, str(ROOT))

K_BASES, S, M, C = 150, 8, 4, 4
KSTEP = 15
Q = 65_536
N_COLS = 16_777_216
TOPK = 20
# DRAM bytes (read + write) of one fused launch of 65,536 reads against
# 2,097,152 index columns (ncu, small enough to capture); traffic grows with
# the column count at a fixed read count, so the bench scales it by N
SMALL_CASE_DRAM_BYTES = 17_403_048_448 + 30_679_040
SMALL_CASE_COLS = 2_097_152
ERR = 0.05
TIE_F16 = 1e-3  # one fp16 step of a score near 1 (2^-10)
GENOME_SEED, READ_SEED = 7, 11
METRIC = "reads/s on 1 B200 at top-20 recall = ref, serving vs plain; p50/p99 latency"


def genome_len(ncols: int) -> int:
    nwin = ncols // 2
    return KSTEP * (nwin - 1) + K_BASES


def make_genome(ncols: int):
    rng = np.random.default_rng(GENOME_SEED)
    return rng.integers(0, 4, size=genome_len(ncols), dtype=np.uint8)


def make_reads(genome: np.ndarray, q: int, seed: int):
    from rotormap import synth
    rng = np.random.default_rng(seed)
    starts = rng.integers(0, genome.size - K_BASES + 1, size=q)
    idx = starts[:, None] + np.arange(K_BASES)[None, :]
    codes = genome[idx]
    hit = rng.random(codes.shape) < ERR
    shift = rng.integers(1, 4, size=codes.shape).astype(np.uint8)
    codes = np.where(hit, (codes + shift) % 4, codes).astype(np.uint8)
    return synth.pack_reads(list(codes), K_BASES), starts


def mapped_fraction(locs: np.ndarray, starts0: np.ndarray, col_start: np.ndarray) -> float:
    """Share of reads whose true window overlaps one of their top-k columns."""
    st = col_start[locs.astype(np.int64) - 1]  # 1-based window starts
    ok = np.abs(st - (starts0[:, None] + 1)) < K_BASES
    return float(ok.any(axis=1).mean())


class Clocks:
    """nvidia-smi samples of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        pw = [float(r[3]) for r in rows if r[3].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w": statistics.median(pw) if pw else None}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# ---------------------------------------------------------------- CPU legs


def cpu_index_sample(genome: np.ndarray, ncols: int, threads: int):
    """The first `ncols` index columns (fwd + rc of the first ncols/2 windows)
    built on the host by the oracle's golden fp64 encoder, scaled e4m3."""
    from oracle import oracle as orc
    from rotormap import synth
    nwin = ncols // 2
    idx = (np.arange(nwin) * KSTEP)[:, None] + np.arange(K_BASES)[None, :]
    codes = genome[idx]
    fw = synth.pack_reads(list(codes), K_BASES)
    rc = synth.pack_reads(list((3 - codes[:, ::-1]).astype(np.uint8)), K_BASES)
    f, _ = orc.rope_f64(np.concatenate([fw, rc]), K_BASES, S, M, C, 0, threads)
    q, sc = orc.quantize_scaled(f.astype(np.float32))
    return q, sc


def cpu_map_sample(words: np.ndarray, Bq, Bs, threads: int):
    """Golden encoder + brute-force scoring of `words` against the column sample."""
    from oracle import oracle as orc
    t0 = time.perf_counter()
    e, _ = orc.rope_f64(words, K_BASES, S, M, C, 0, threads)
    a8, sa = orc.quantize_scaled(e.astype(np.float32))
    orc.topk_e4m3(a8, Bq, TOPK, 2, sa, Bs, threads)
    return time.perf_counter() - t0


def cpu_baseline(genome, reads_words, threads: int, budget_s: float = 12.0):
    sample_cols = 1 << 18
    Bq, Bs = cpu_index_sample(genome, sample_cols, threads)
    t_cal = cpu_map_sample(reads_words[:8], Bq, Bs, threads)
    nr = int(max(8, min(4096, 8 * budget_s / max(t_cal, 1e-3))))
    t = cpu_map_sample(reads_words[:nr], Bq, Bs, threads)
    value = nr * (sample_cols / N_COLS) / t
    return {"value": value, "unit": "reads/s", "cores": threads, "kind": "port",
            "sample": f"{nr} reads x {sample_cols} of {N_COLS} index columns (golden fp64 encode + "
                      f"brute-force scaled-e4m3 scores + top-{TOPK}), reads/s scaled to the full index",
            "seconds": t}


def run_reference(args):
    """--impl reference: the CPU restatement of the reference path (the
    reference itself is Julia and is not installed here), same metric."""
    threads = os.cpu_count() or 1
    genome = make_genome(N_COLS)
    words, _ = make_reads(genome, 4096, READ_SEED)
    sample_cols = 1 << 18
    Bq, Bs = cpu_index_sample(genome, sample_cols, threads)
    per = 64
    t_cal = cpu_map_sample(words[:8], Bq, Bs, threads)
    per = int(max(8, min(2048, 8 * 8.0 / max(t_cal, 1e-3))))  # ~8 s per step
    for i in range(args.warmup):
        cpu_map_sample(words[:8], Bq, Bs, threads)
    ts = []
    for i in range(args.steps):
        lo = (i * per) % (words.shape[0] - per)
        ts.append(cpu_map_sample(words[lo:lo + per], Bq, Bs, threads))
    tot = sum(ts)
    value = per * args.steps * (sample_cols / N_COLS) / tot
    line = {"metric": METRIC, "value": value, "unit": "reads/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 encode / e4m3 scores", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "kernel microbench: Q=65536 x 150bp reads vs N=16777216 index columns",
                       "sample_reads_per_step": per, "sample_cols": sample_cols, "k": TOPK},
            "cpu_baseline": {"value": value, "unit": "reads/s", "cores": threads, "kind": "port",
                             "sample": f"{per} reads x {sample_cols} columns per step, scaled to N"},
            "e2e": {"value": value, "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def fp64_check(re, idx, genome_dev, words_dev, locs8, vals8, n_sample: int, seed: int):
    """Top-20 recall and score error of the fp8 search against the exact
    FP64 search over all index columns (the GPU check kernel, windows
    re-encoded with the golden fp64 encoder) on `n_sample` sampled reads."""
    import torch
    import rotormap as rm
    rng = np.random.default_rng(seed)
    nq = words_dev.shape[0]
    samp = np.sort(rng.choice(nq, size=min(n_sample, nq), replace=False))
    ds = torch.from_numpy(samp).to(words_dev.device)
    meta = rm.DeviceMeta(idx, genome=genome_dev)
    cand = locs8[ds].contiguous()
    t0 = time.perf_counter()
    v64, l64, c64 = rm.check_fp64(re, meta, words_dev[ds].contiguous(), cand)
    secs = time.perf_counter() - t0
    l8, l64, v8, c64 = cand.cpu().numpy(), l64.cpu().numpy(), vals8[ds].cpu().numpy(), c64.cpu().numpy()
    rec = float(np.mean([len(set(a) & set(b)) / TOPK for a, b in zip(l8, l64)]))
    err = np.abs(v8.astype(np.float64) - c64)
    del meta
    return {"sampled_rows": int(samp.size), "seconds": secs, "top20_recall_fp8_vs_fp64": rec,
            "score_abs_err_fp8": {"max": float(err.max()), "mean": float(err.mean())}}


# ---------------------------------------------------------------- serving leg


def serving_leg(dev, n_requests: int = 16, seed: int = 31, fp64_sample: int = 0, kernel_tflops=None,
                rows: int = 131072):
    """Serving form vs the plain batch path at human-scale geometry: 3.1 Gbp
    genome of 24 records (lengths U[50, 250] Mbp rescaled, GC 41%, 5% N runs),
    fwd + rc windows at k = 150, kstep = 1880 -> ~3.3M columns (~6.3 GiB e4m3),
    Poisson arrivals of requests of U{1..100,000} reads with substitution
    rates U[0, 0.10], offered at 1.5x the fused kernel's capacity (the
    headline leg's measured TFLOP/s when given, else 2.2 PFLOP/s), so the
    server stays loaded.  Same arrival schedule for every path."""
    import torch
    import rotormap as rm
    from rotormap import serving, synth
    re = rm.RopeEncoder(k=K_BASES, s=S, m=M, c=C)
    lengths = synth.genome_lengths(3_100_000_000, 24, 50e6, 250e6, seed)
    words, woff, nbases, runs = synth.random_genome_packed(lengths, seed=seed, gc=0.41, n_frac=0.05, device=dev)
    heads = [f">chr{i + 1} synthetic human-scale record" for i in range(24)]
    idx = rm.build_index_packed(re, words, heads, woff, nbases, 1880)
    rng = np.random.default_rng(seed + 1)
    sizes = rng.integers(1, 100_001, n_requests)
    errs = rng.uniform(0.0, 0.10, n_requests)
    reqs, truth = [], []
    for i, n in enumerate(sizes):
        recs, offs = synth.sample_positions(nbases, runs, int(n), K_BASES, seed + 10 + i)
        reqs.append(synth.extract_reads_packed(words, woff, recs, offs, K_BASES, float(errs[i]), seed + 10 + i))
        truth.append((recs, offs))
    torch.cuda.empty_cache()
    total = int(sizes.sum())
    # arrivals: Poisson, mean gap = mean request / (1.5 x the fused kernel's capacity)
    flop_per_read = 2.0 * re.rdim * idx.N
    cap_flops = kernel_tflops * 1e12 if kernel_tflops else 2.2e15
    cap_est = cap_flops / flop_per_read
    gaps = rng.exponential(float(sizes.mean()) / (1.5 * cap_est), n_requests)
    arrivals = np.concatenate([[0.0], np.cumsum(gaps[1:])])

    def replay(t0):
        def wait(t):
            d = t0 + t - time.perf_counter()
            if d > 0:
                time.sleep(d)
        return wait

    def stats(done_times, t0):
        lat = np.array([d - (t0 + a) for d, a in zip(done_times, arrivals)])
        span = max(done_times) - t0
        return {"reads_per_s": total / span, "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "span_s": span}

    out = {"workload": f"3.1 Gbp genome (24 records, GC 41%, 5% N), k=150 kstep=1880 -> N={idx.N} "
                       f"columns ({idx.N * re.rdim / 2**30:.2f} GiB e4m3), {n_requests} Poisson requests "
                       f"of U{{1..100000}} reads (total {total}), subs U[0,0.10], top-20, f16 scores, "
                       f"offered at 1.5 x {cap_flops / 1e15:.2f} PFLOP/s, batches of up to {rows} reads",
           "index_cols": idx.N, "requests": n_requests, "reads": total}
    # serving form (fused kernel, continuous batching)
    eng = rm.TopKEngine(idx.embeds8, k=TOPK, rows_cap=rows, score="f16")
    srv = serving.MappingServer(eng, re)
    srv.submit(reqs[0][:64]).result(300)  # warm-up
    clk = Clocks(dev.index if dev.index is not None else 0)
    clk.start()
    t0 = time.perf_counter()
    wait = replay(t0)
    hs = []
    for a, w in zip(arrivals, reqs):
        wait(a)
        hs.append(srv.submit(w, t_arrival=t0 + a))
    res = [h.result(600) for h in hs]
    done_times = [h.t_done for h in hs]  # results in host memory (CLOCK_MONOTONIC = perf_counter's clock)
    clocks = clk.stop()
    sst = srv.stats()
    srv.close()
    out["serving"] = stats(done_times, t0)
    out["serving"]["batches"] = sst.batches
    out["serving"]["loop"] = "native (r2m_server_*)"
    out["serving"]["tflops"] = total * flop_per_read / out["serving"]["span_s"] / 1e12
    # tensor-pipe utilisation over the whole span (arrival gaps, encodes and
    # merges included): achieved / (16384 dense fp8 FLOP per SM per clock x
    # SMs x the median SM clock sampled during the span)
    out["serving"]["clocks"] = clocks
    if clocks.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        out["serving"]["tensor_pipe_est"] = out["serving"]["tflops"] / (16384.0 * sms * clocks["sm_mhz"] * 1e-6)
    # plain batch path, reference engine structure (cuBLASLt fp8 + segmented top-k, batch 8192)
    peng = rm.PlainEngine(idx.embeds8, k=TOPK, w=65536, rows_cap=8192)
    serving.plain_map(peng, re, [(0.0, reqs[0][:64])], batch=8192)
    t0 = time.perf_counter()
    pres = serving.plain_map(peng, re, list(zip(arrivals, reqs)), batch=8192, clock=replay(t0))
    out["plain_reference_engine"] = stats([p[0] for p in pres], t0)
    peng.close()
    # plain batch path with the fused kernel (fixed 8192 batches, one request at a time)
    t0 = time.perf_counter()
    fres = serving.plain_map(eng, re, list(zip(arrivals, reqs)), batch=8192, clock=replay(t0))
    out["plain_fused_kernel"] = stats([p[0] for p in fres], t0)
    eng.close()
    out["serving_vs_plain"] = out["serving"]["reads_per_s"] / out["plain_reference_engine"]["reads_per_s"]
    # top-20 recall against the reference-structured engine.  That engine
    # keeps an arbitrary one of tied locations (its segmented top-k), so a
    # served location that is not in its list counts as recalled when it ties
    # the list's 20th value within one fp16 step (both paths round fp32 sums
    # to fp16); `untied_misses` counts the served locations that are neither.
    sv = np.concatenate([v for v, _ in res]).astype(np.float32)
    sl = np.concatenate([l for _, l in res])
    pv = np.concatenate([p[1] for p in pres]).astype(np.float32)
    pl = np.concatenate([p[2] for p in pres])
    inset = np.zeros(sl.shape, bool)
    for r0 in range(0, sl.shape[0], 65536):
        inset[r0:r0 + 65536] = (sl[r0:r0 + 65536, :, None] == pl[r0:r0 + 65536, None, :]).any(axis=2)
    tied = ~inset & (sv >= pv[:, -1:] - TIE_F16)
    out["top20_recall_vs_plain_reference"] = float((inset | tied).mean())
    out["top20_set_overlap_vs_plain_reference"] = float(inset.mean())
    out["untied_misses"] = int((~inset & ~tied).sum())
    out["tie_tolerance"] = TIE_F16
    # provenance: a read maps if a top-20 window overlaps its true position
    hit = 0
    recmap = idx.col_rec
    for (v, l), (recs, offs) in zip(res, truth):
        c = l.astype(np.int64) - 1
        ok = (recmap[c] == recs[:, None]) & (np.abs(idx.starts[c] - (offs[:, None] + 1)) < K_BASES)
        hit += int(ok.any(axis=1).sum())
    out["mapped_frac_top20"] = hit / total
    if fp64_sample > 0:
        W = re.words
        allw = torch.from_numpy(np.concatenate(reqs).reshape(-1).view(np.int32)).to(dev).view(-1, W)
        out["fp64_check"] = fp64_check(re, idx, words, allw, torch.from_numpy(sl).to(dev),
                                       torch.from_numpy(sv).to(dev), fp64_sample, seed + 5)
        del allw
    del idx, words
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------- precision leg


def precision_leg(dev, n_reads: int, n_sample: int, seed: int = 51):
    """Precision form on the 100 Mbp configuration: 10 records x 10 Mbp,
    GC 41%, 1% N runs of 100..10,000 bp, k = 150, kstep = 15 (fwd + rc,
    ~13.3M columns, per-column scaled e4m3); reads of 150 bp with 5% iid
    substitutions; fp8 top-64 -> FP32 rescoring -> top-20; FP64 check on
    `n_sample` sampled rows (score error, top-20 recall)."""
    import torch
    import rotormap as rm
    from rotormap import synth
    re = rm.RopeEncoder(k=K_BASES, s=S, m=M, c=C)
    lengths = np.full(10, 10_000_000, np.int64)
    words, woff, nbases, runs = synth.random_genome_packed(lengths, seed=seed, gc=0.41, n_frac=0.01,
                                                           run_min=100, run_max=10_000, device=dev)
    heads = [f">rec{i + 1} synthetic 10 Mbp" for i in range(10)]
    t0 = time.perf_counter()
    idx = rm.build_index_packed(re, words, heads, woff, nbases, KSTEP, scaled=True)
    t_index = time.perf_counter() - t0
    meta = rm.DeviceMeta(idx, genome=words)
    recs, offs = synth.sample_positions(nbases, runs, n_reads, K_BASES, seed + 1)
    rw = synth.extract_reads_packed(words, woff, recs, offs, K_BASES, ERR, seed + 1)
    dw = torch.from_numpy(rw.view(np.int32)).to(dev)
    eng = rm.TopKEngine(idx.embeds8, k=64, rows_cap=n_reads, score="scaled", scaleB=idx.scales)
    rm.map_precise(eng, re, meta, dw[:256])  # warm-up
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    st = torch.cuda.current_stream()
    e0.record(st)
    nb = n_reads
    a8, sa = eng.a8[:nb], eng.scaleA[:nb]
    norms = torch.empty((nb, M), dtype=torch.float32, device=dev)
    rm.encode_frag_real_batch(a8, norms, re, dw.reshape(-1), 0, sa)
    v8, l8 = eng.search(a8, nb, sa)
    e1.record(st)
    v32, l32 = rm.rescore_fp32(re, meta, dw, l8, TOPK)
    e2.record(st)
    torch.cuda.synchronize()
    t_fp8, t_resc = e0.elapsed_time(e1) / 1e3, e1.elapsed_time(e2) / 1e3
    # FP64 check on sampled rows
    rng = np.random.default_rng(seed + 2)
    samp = np.sort(rng.choice(n_reads, size=n_sample, replace=False))
    ds = torch.from_numpy(samp).to(dev)
    cand = torch.cat([l8[ds][:, :TOPK], l32[ds]], dim=1).contiguous()
    t0 = time.perf_counter()
    v64, l64, c64 = rm.check_fp64(re, meta, dw[ds].contiguous(), cand)
    t_check = time.perf_counter() - t0
    l8s, l32s, l64 = l8[ds][:, :TOPK].cpu().numpy(), l32[ds].cpu().numpy(), l64.cpu().numpy()
    v8s, v32s, c64 = v8[ds][:, :TOPK].cpu().numpy(), v32[ds].cpu().numpy(), c64.cpu().numpy()
    rec = lambda a, b: float(np.mean([len(set(x) & set(y)) / TOPK for x, y in zip(a, b)]))
    err8 = np.abs(v8s - c64[:, :TOPK])
    err32 = np.abs(v32s - c64[:, TOPK:])
    l32a = l32.cpu().numpy()
    c = l32a.astype(np.int64) - 1
    ok = (idx.col_rec[c] == recs[:, None]) & (np.abs(idx.starts[c] - (offs[:, None] + 1)) < K_BASES)
    out = {"workload": f"100 Mbp genome (10 x 10 Mbp, GC 41%, 1% N runs), k=150 kstep=15 -> N={idx.N} columns "
                       f"(scaled e4m3), {n_reads} reads x 150 bp (5% subs), fp8 top-64 -> FP32 rescore -> top-20",
           "index_cols": idx.N, "reads": n_reads, "index_build_s": t_index,
           "fp8_search_s": t_fp8, "rescore_s": t_resc,
           "reads_per_s": n_reads / (t_fp8 + t_resc),
           "fp64_check": {"sampled_rows": n_sample, "seconds": t_check,
                          "top20_recall_fp8": rec(l8s, l64), "top20_recall_fp32_rescored": rec(l32s, l64),
                          "score_abs_err_fp8": {"max": float(err8.max()), "mean": float(err8.mean())},
                          "score_abs_err_fp32": {"max": float(err32.max()), "mean": float(err32.mean())}},
           "mapped_frac_top20": float(ok.any(axis=1).mean())}
    eng.close()
    del idx, meta, words, eng
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------- batching leg


def batching_leg(dev, n_requests: int, seed: int = 61):
    """Batching form on the 100 Mbp genome indexed at k = 100, kstep = 10
    (~20M columns): requests with log-uniform read counts on [1, 50,000],
    lognormal read lengths (median 150, clipped to [100, 250], trimmed to the
    first k = 100 bases like the reference reader), substitution rate
    U[0, 0.15].  One ragged launch per request set (graph-captured,
    autotuned) vs mapping the requests one at a time."""
    import torch
    import rotormap as rm
    from rotormap import synth
    kb = 100
    re = rm.RopeEncoder(k=kb, s=S, m=M, c=C)
    lengths = np.full(10, 10_000_000, np.int64)
    words, woff, nbases, runs = synth.random_genome_packed(lengths, seed=51, gc=0.41, n_frac=0.01,
                                                           run_min=100, run_max=10_000, device=dev)
    idx = rm.build_index_packed(re, words, [f">rec{i + 1}" for i in range(10)], woff, nbases, 10)
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(0, np.log(50_000), n_requests)).astype(np.int64)
    lens = np.clip(np.exp(rng.normal(np.log(150), 0.25, n_requests)), 100, 250).astype(int)
    errs = rng.uniform(0, 0.15, n_requests)
    reqs = []
    for i, n in enumerate(counts):
        recs, offs = synth.sample_positions(nbases, runs, int(n), int(lens[i]), seed + i)
        reqs.append(synth.extract_reads_packed(words, woff, recs, offs, kb, float(errs[i]), seed + i))
    del words
    total = int(counts.sum())
    eng = rm.TopKEngine(idx.embeds8, k=TOPK, rows_cap=rm.bucket_rows(total), score="f16")
    tuner = rm.Autotuner()  # no cache file: this run pays the tuning
    b = rm.RaggedBatcher(eng, re, total, tuner=tuner, use_graphs=True)
    t0 = time.perf_counter()
    b.run(reqs)  # tune + capture + first replay
    t_first = time.perf_counter() - t0
    t0 = time.perf_counter()
    res = b.run(reqs)
    t_ragged = time.perf_counter() - t0
    tuned = {k: tuner.last[k] for k in ("splits", "ctas", "kernel", "epilogue", "pace", "kt")}
    default = {"splits": 0, "ctas": 0, "kernel": "auto", "epilogue": "auto", "pace": 0, "kt": 0}
    if tuned == default:
        t_untuned = t_ragged  # the tuner kept the built-in schedule
    else:  # the same graph-replayed launch with the built-in schedule
        eng.set_tuning(0, 0, kernel="auto", epilogue="auto", pace=0, kt=0)
        bu = rm.RaggedBatcher(eng, re, total, tuner=None, use_graphs=True)
        bu.run(reqs)
        t0 = time.perf_counter()
        ru = bu.run(reqs)
        t_untuned = time.perf_counter() - t0
        assert all(np.array_equal(a[1], c[1]) for a, c in zip(res, ru)), "schedules changed the results"
        del bu
    # one request at a time (encode + search + D2H per request, synchronous)
    eng.set_tuning(0, 0, kernel="auto", epilogue="auto", pace=0, kt=0)
    st = torch.cuda.current_stream()
    t0 = time.perf_counter()
    for w in reqs:
        d = torch.from_numpy(w.reshape(-1).view(np.int32)).to(dev, non_blocking=True)
        a8, nrm = rm.encode_frag_real_batch_alloc(torch.uint8, re, d)
        v, l = eng.search(a8)
        v.cpu(), l.cpu()
    torch.cuda.synchronize()
    t_each = time.perf_counter() - t0
    out = {"workload": f"100 Mbp genome at k=100 kstep=10 -> N={idx.N} columns, {n_requests} requests "
                       f"(log-uniform 1..50000 reads, total {total}), lengths lognormal median 150 in [100,250] "
                       f"trimmed to 100, subs U[0,0.15], top-20, f16 scores",
           "index_cols": idx.N, "requests": n_requests, "reads": total,
           "ragged_graph_reads_per_s": total / t_ragged, "per_request_reads_per_s": total / t_each,
           "speedup": t_each / t_ragged, "first_run_s": t_first, "launch_sets": 1,
           "untuned_reads_s": total / t_untuned, "tuned_vs_untuned": t_untuned / t_ragged,
           "tuning_cost_frac": tuner.last["tune_s"] / t_ragged,
           "autotuned": {"chosen": tuned, "tune_s": tuner.last["tune_s"], "proxy_cols": tuner.last["proxy_cols"],
                         "proxy_default_ms": tuner.last["default_ms"], "proxy_best_ms": tuner.last["ms"],
                         "candidates": tuner.log}}
    eng.close()
    del idx, eng, b
    torch.cuda.empty_cache()
    return out


def compact_leg(dev, ncols: int = 4_194_304, chunk: int = 1 << 20, seed: int = 81):
    """Host-ring engine: an index of `ncols` scaled-e4m3 columns (k = 150,
    stride 15, from a seeded random genome) kept in page-locked host memory
    and streamed through a 3-slot device ring of `chunk` columns per search,
    against the same index resident in HBM.  Batches of 65,536 and 8,192
    reads; CUDA-event timing, 3 searches after one warm-up; results checked
    equal to the resident engine's."""
    import torch

    import rotormap as rm
    from rotormap import synth
    re = rm.RopeEncoder(k=K_BASES, s=S, m=M, c=C)
    nbases = (ncols // 2 - 1) * KSTEP + K_BASES
    words, woff, nb, runs = synth.random_genome_packed([nbases], seed=seed, gc=0.41, device=dev)
    idx = rm.build_index_packed(re, words, [">g"], woff, nb, KSTEP, scaled=True)
    recs, offs = synth.sample_positions(nb, runs, 65_536, K_BASES, seed)
    rw = synth.extract_reads_packed(words, woff, recs, offs, K_BASES, np.full(len(recs), 0.05), seed)
    del words
    Bh = idx.embeds8.cpu().numpy()
    sb = idx.scales if isinstance(idx.scales, torch.Tensor) else torch.from_numpy(np.asarray(idx.scales))
    sb = sb.to(dev)
    dw = torch.from_numpy(np.ascontiguousarray(rw).view(np.int32)).to(dev)
    a8, _, sa = rm.encode_frag_real_batch_alloc(torch.uint8, re, dw, scaled=True)
    out = {"workload": f"{idx.N} columns ({Bh.nbytes / 2**30:.2f} GiB e4m3) in host memory, ring of 3 x {chunk} "
                       f"columns; scaled scores, top-{TOPK}", "index_cols": idx.N, "chunk_cols": chunk}
    res = rm.TopKEngine(idx.embeds8, k=TOPK, rows_cap=65_536, score="scaled", scaleB=sb)
    t0 = time.perf_counter()
    ring = rm.CompactEngine(Bh, k=TOPK, rows_cap=65_536, score="scaled", scaleB=sb, chunk_cols=chunk, depth=3,
                            pin=True)
    out["create_s"] = time.perf_counter() - t0
    out["pinned"] = ring.pinned
    out["chunks"] = ring.chunks
    st = torch.cuda.current_stream(dev)

    def timed(eng, nq):
        eng.search(a8[:nq], nq, sa[:nq])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(3):
            v, l = eng.search(a8[:nq], nq, sa[:nq])
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / 3, v, l

    # the same host index with half of it kept on the device (2 of 4 chunks)
    half = rm.CompactEngine(Bh, k=TOPK, rows_cap=65_536, score="scaled", scaleB=sb, chunk_cols=chunk, depth=3,
                            pin=True, resident_chunks=2)
    for nq in (65_536, 8_192):
        ms_r, v0, l0 = timed(res, nq)
        ms_c, v1, l1 = timed(ring, nq)
        ms_h, v2, l2 = timed(half, nq)
        out[f"q{nq}"] = {"resident_reads_per_s": nq / ms_r * 1e3, "ring_reads_per_s": nq / ms_c * 1e3,
                         "ring_over_resident": ms_r / ms_c, "ring_h2d_GBps": Bh.nbytes / ms_c / 1e6,
                         "half_resident_reads_per_s": nq / ms_h * 1e3, "half_resident_over_resident": ms_r / ms_h,
                         "identical": bool(torch.equal(v0, v1) and torch.equal(l0, l1)
                                           and torch.equal(v0, v2) and torch.equal(l0, l2))}
    half.close()
    ring.close()
    res.close()
    del idx, res, ring, half, Bh, a8, sa, dw, sb
    torch.cuda.empty_cache()
    return out


def gemm_bar_leg(dev, seconds: float = 2.0):
    """The GEMM bar of the reference's production engine: cuBLASLt's fp8
    GEMM (through torch._scaled_mm, which calls it) at the engine's chunk
    shape -- M = 8,192 reads, K = 2,048, N = 65,536 index columns, e4m3
    operands, fp32 accumulation, fp16 C (RotorMap/gemm/fp8_lt.jl:95-168) --
    without any top-k.  Timed as a burst (20 calls) and as a loop of about
    `seconds` (the power-capped regime the fused kernel's ~1.8 s launches
    run in).  A measurement of the library, not part of this path."""
    import torch
    M, K, N = 8192, 2048, 65536
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    a = (torch.rand((M, K), generator=g, device=dev) * 2 - 1).to(torch.float8_e4m3fn)
    b = (torch.rand((N, K), generator=g, device=dev) * 2 - 1).to(torch.float8_e4m3fn)
    one = torch.ones((), dtype=torch.float32, device=dev)

    def run():
        return torch._scaled_mm(a, b.t(), scale_a=one, scale_b=one, out_dtype=torch.float16)

    for _ in range(3):
        run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(20):
        run()
    e1.record()
    e1.synchronize()
    burst_ms = e0.elapsed_time(e1) / 20
    reps = max(20, int(seconds * 1e3 / max(burst_ms, 1e-3)))
    clk = Clocks(dev.index if dev.index is not None else 0)
    clk.start()
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    e1.synchronize()
    c = clk.stop()
    sus_ms = e0.elapsed_time(e1) / reps
    flop = 2.0 * M * K * N
    sus = flop / sus_ms / 1e9
    return {"library": "cuBLASLt fp8 via torch._scaled_mm", "shape": {"M": M, "K": K, "N": N},
            "out": "fp16", "burst_ms": burst_ms, "burst_tflops": flop / burst_ms / 1e9,
            "sustained_ms": sus_ms, "sustained_tflops": sus, "sustained_calls": reps,
            "sustained_clocks": c,
            "tflops_per_w": sus / c["power_w"] if c.get("power_w") else None}


def map_leg(dev, n_reads: int = 400_000, ncols: int = 1_048_576, seed: int = 91):
    """run_map end to end (RotorMap/tools/map.jl): a FASTA file of n_reads
    150 bp reads (5% substitutions, provenance headers) sampled from a seeded
    genome, mapped against its index of `ncols` columns (k = 150, stride 15,
    f16 scores, top-20) and written as the match table -- FASTA parse (GPU or
    host reader), encode, fused search and the threaded table writer
    overlapped with the next batch.  Compared with the search alone."""
    import tempfile

    import torch

    import rotormap as rm
    from rotormap import synth
    re = rm.RopeEncoder(k=K_BASES, s=S, m=M, c=C)
    nbases = (ncols // 2 - 1) * KSTEP + K_BASES
    words, woff, nb, runs = synth.random_genome_packed([nbases], seed=seed, gc=0.41, device=dev)
    idx = rm.build_index_packed(re, words, [">chr1 synthetic"], woff, nb, KSTEP)
    recs, offs = synth.sample_positions(nb, runs, n_reads, K_BASES, seed)
    rw = synth.extract_reads_packed(words, woff, recs, offs, K_BASES, 0.05, seed)
    del words
    j = np.arange(K_BASES)
    codes = ((rw[:, j >> 4] >> (2 * (j & 15)).astype(np.uint32)) & 3).astype(np.uint8)
    letters = synth.LETTERS[codes]
    raw = b"".join(b">read_%d start=%d len=150 src=chr1\n" % (i + 1, offs[i] + 1) + letters[i].tobytes() + b"\n"
                   for i in range(n_reads))
    out = {"workload": f"{n_reads} reads x 150 bp FASTA ({len(raw)} bytes) vs {idx.N} columns, f16 top-20, "
                       f"batches of 65,536; table of {n_reads * TOPK} lines"}
    with tempfile.TemporaryDirectory() as tdir:
        fa = os.path.join(tdir, "reads.fa")
        with open(fa, "wb") as f:
            f.write(raw)
        warm = os.path.join(tdir, "warm.maps")
        rm.run_map(idx, fa, warm, topk=TOPK, batch_size=65_536)
        # each ~540 MB table is deleted before the next run, so the next run
        # does not write while the kernel still flushes the previous file
        os.remove(warm)
        for reader in ("device", "host"):
            dst = os.path.join(tdir, f"{reader}.maps")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            n = rm.run_map(idx, fa, dst, topk=TOPK, batch_size=65_536, reader=reader)
            dt = time.perf_counter() - t0
            with open(dst, "rb") as f:
                lines = sum(1 for _ in f)
            os.remove(dst)
            out[f"run_map_{reader}_reader"] = {"seconds": dt, "reads_per_s": n / dt, "lines": lines}
    eng = rm.TopKEngine(idx.embeds8, k=TOPK, rows_cap=65_536)
    a8, _ = rm.encode_frag_real_batch_alloc(torch.uint8, re, torch.from_numpy(rw[:65_536].view(np.int32)).to(dev))
    eng.search(a8)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        eng.search(a8)
    torch.cuda.synchronize()
    out["search_only_reads_per_s"] = 3 * 65_536 / (time.perf_counter() - t0)
    eng.close()
    del idx, eng, a8
    torch.cuda.empty_cache()
    return out


def fasta_leg(dev, n_reads: int = 400_000, seed: int = 71):
    """Reads-side FASTA parsing: the native host reader (all cores) against
    the GPU reader, on a FASTA of n_reads 150 bp reads with provenance-style
    headers.  Device figures: the C entry on bytes already in HBM (CUDA
    events, 5 calls) and the Python API from host bytes (H2D of the file,
    the parse, words left on the device, headers back to the host)."""
    import ctypes

    import torch

    import rotormap as rm
    from rotormap import synth
    from rotormap._lib import check, lib, ptr, stream_handle
    rng = np.random.default_rng(seed)
    codes = rng.integers(0, 4, (n_reads, K_BASES), dtype=np.uint8)
    pos = rng.integers(1, 100_000_000, n_reads)
    letters = synth.LETTERS[codes]
    raw = b"".join(b">read_%d start=%d len=150 src=chr1\n" % (i, pos[i]) + letters[i].tobytes() + b"\n"
                   for i in range(n_reads))
    nbytes = len(raw)
    threads = os.cpu_count() or 1
    rm.fasta_reads(raw, k=K_BASES, parts=threads)
    t_hosts = []
    for _ in range(5):  # the box's host cores are shared: best and median of 5
        t0 = time.perf_counter()
        h = rm.fasta_reads(raw, k=K_BASES, parts=threads)
        t_hosts.append(time.perf_counter() - t0)
    t_host = min(t_hosts)
    d_raw = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(dev)
    for _ in range(3):
        g = rm.fasta_reads_device(raw, k=K_BASES, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g = rm.fasta_reads_device(raw, k=K_BASES, device=dev)
    torch.cuda.synchronize()
    t_api = time.perf_counter() - t0
    same = g.heads == h.heads and np.array_equal(g.words.cpu().numpy().view(np.uint32), h.words)
    L = lib()
    hd = ctypes.c_void_p()
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(5):
        check(L.r2m_fasta_reads_device(ptr(d_raw), nbytes, K_BASES, stream_handle(st), ctypes.byref(hd)))
        L.r2m_dreads_free(hd)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / 5
    del d_raw, g
    torch.cuda.empty_cache()
    return {"workload": f"{n_reads} reads of 150 bp, {nbytes} bytes of FASTA", "bytes": nbytes,
            "host_native_s": t_host, "host_native_GBps": nbytes / t_host / 1e9,
            "host_native_median_s": float(np.median(t_hosts)), "host_threads": threads,
            "device_c_entry_ms": ms, "device_c_entry_GBps": nbytes / ms / 1e6,
            "device_api_from_host_s": t_api, "device_api_from_host_GBps": nbytes / t_api / 1e9,
            "identical_to_host_reader": bool(same)}


# ---------------------------------------------------------------- GPU leg


def _r(x, nd=4):
    return None if x is None else float(f"{x:.{nd}g}")


def summary(line: dict) -> dict:
    """The figures of every leg in one compact object (printed last)."""
    out = {"headline_reads_s": _r(line["value"]), "e2e_reads_s": _r(line["e2e"]["value"]),
           "gemm_tflops": _r(line["roofline"]["achieved"]), "gemm_frac_of_2x_bf16": _r(line["roofline"]["frac"], 3),
           "encoder_gbs": _r(line["encoder"]["achieved_gbs"]),
           "encoder_frac_hbm": _r(line["encoder"]["achieved_gbs"] / line["encoder"]["peak_gbs"], 3),
           "encoder_alone_gbs": _r(line["encoder"]["alone_gbs"]),
           "encoder_alone_frac_hbm": _r(line["encoder"]["alone_gbs"] / line["encoder"]["peak_gbs"], 3)}
    if line.get("fp64_check"):
        out["C1_fp64_recall"] = _r(line["fp64_check"]["top20_recall_fp8_vs_fp64"], 4)
        out["C1_fp64_err_max"] = _r(line["fp64_check"]["score_abs_err_fp8"]["max"], 3)
    if "tensor_pipe" in line["roofline"]:
        out["tensor_pipe_est"] = _r(line["roofline"]["tensor_pipe"].get("est_active_frac"), 3)
    sv = line.get("serving")
    if sv:
        out["C4_serving"] = {"reads_s": _r(sv["serving"]["reads_per_s"]), "p50_s": _r(sv["serving"]["p50_s"], 3),
                             "p99_s": _r(sv["serving"]["p99_s"], 3),
                             "vs_plain_reference_engine": _r(sv["serving_vs_plain"], 3),
                             "vs_plain_fused_kernel": _r(sv["serving"]["reads_per_s"] /
                                                         sv["plain_fused_kernel"]["reads_per_s"], 3),
                             "recall_vs_plain_ties": _r(sv["top20_recall_vs_plain_reference"], 6),
                             "untied_misses": sv["untied_misses"], "reads": sv["reads"],
                             "tflops": _r(sv["serving"]["tflops"]),
                             "tensor_pipe_est": _r(sv["serving"].get("tensor_pipe_est"), 3)}
        if sv.get("fp64_check"):
            out["C4_serving"]["fp64_recall"] = _r(sv["fp64_check"]["top20_recall_fp8_vs_fp64"], 4)
            out["C4_serving"]["fp64_err_max"] = _r(sv["fp64_check"]["score_abs_err_fp8"]["max"], 3)
    pr = line.get("precision")
    if pr:
        fc = pr["fp64_check"]
        out["C2_precision"] = {"reads": pr["reads"], "reads_s": _r(pr["reads_per_s"]),
                               "sampled_rows": fc["sampled_rows"],
                               "recall_fp8": _r(fc["top20_recall_fp8"], 4),
                               "recall_fp32": _r(fc["top20_recall_fp32_rescored"], 4),
                               "err_fp8_max": _r(fc["score_abs_err_fp8"]["max"], 3),
                               "err_fp32_max": _r(fc["score_abs_err_fp32"]["max"], 3)}
    bt = line.get("batching")
    if bt:
        out["C3_batching"] = {"requests": bt["requests"], "reads": bt["reads"],
                              "ragged_reads_s": _r(bt["ragged_graph_reads_per_s"]),
                              "per_request_reads_s": _r(bt["per_request_reads_per_s"]),
                              "speedup": _r(bt["speedup"], 3), "first_run_s": _r(bt["first_run_s"], 3)}
        for key in ("untuned_reads_s", "tuned_vs_untuned", "tuning_cost_frac"):
            if key in bt:
                out["C3_batching"][key] = _r(bt[key], 3)
    fa = line.get("fasta_reader")
    if fa:
        out["fasta_GBps"] = {k[:-5]: _r(v, 3) for k, v in fa.items()
                             if isinstance(v, (int, float)) and k.endswith("_GBps")}
    if line.get("cpu_baseline"):
        out["cpu_baseline_reads_s"] = _r(line["cpu_baseline"]["value"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ncols", type=int, default=N_COLS)
    ap.add_argument("--reads", type=int, default=Q)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--splits", type=int, default=0, help="force the column split count (0 = auto)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-vs-plain leg")
    ap.add_argument("--serving-rows", type=int, default=131072,
                    help="largest GPU batch of the serving loop (131,072: fewer, longer launches -- tensor pipe "
                         "0.71 vs 0.68 at 65,536, p50 latency 1.6 vs 1.3 s)")
    ap.add_argument("--requests", type=int, default=16, help="requests in the serving leg")
    ap.add_argument("--no-precision", action="store_true", help="skip the precision leg")
    ap.add_argument("--no-batching", action="store_true", help="skip the batching leg")
    ap.add_argument("--no-fasta", action="store_true", help="skip the FASTA reader leg")
    ap.add_argument("--no-compact", action="store_true", help="skip the host-ring engine leg")
    ap.add_argument("--no-map", action="store_true", help="skip the run_map end-to-end leg")
    ap.add_argument("--no-gemm-bar", action="store_true", help="skip the cuBLASLt fp8 GEMM bar")
    ap.add_argument("--batching-requests", type=int, default=256)
    ap.add_argument("--precision-reads", type=int, default=1_000_000)
    ap.add_argument("--precision-sample", type=int, default=10_000)
    ap.add_argument("--fp64-sample", type=int, default=1000,
                    help="reads of the headline and serving legs checked against the exact FP64 search")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch
    import torch.distributed as dist

    import rotormap as rm

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    re = rm.RopeEncoder(k=K_BASES, s=S, m=M, c=C)
    genome = make_genome(args.ncols)
    pack = rm.pack_records([">synthetic_genome seed=7"], [genome])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    idx = rm.build_index(re, "synthetic", kstep=KSTEP, scaled=True, pack=pack)
    torch.cuda.synchronize()
    t_index = time.perf_counter() - t0
    N = idx.N
    words, starts0 = make_reads(genome, args.reads, READ_SEED + 1000 * rank)
    nq = words.shape[0]
    dev = torch.device("cuda", local)
    d_words = torch.from_numpy(words.reshape(-1).view(np.int32)).to(dev)
    eng = rm.TopKEngine(idx.embeds8, k=TOPK, rows_cap=nq, score="scaled", scaleB=idx.scales, timing=True,
                        splits=args.splits)
    a8, sa = eng.a8[:nq], eng.scaleA[:nq]
    norms = torch.empty((nq, M), dtype=torch.float32, device=dev)
    d_val = torch.empty((nq, TOPK), dtype=torch.float32, device=dev)
    d_loc = torch.empty((nq, TOPK), dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev)
    enc_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def step():
        enc_ev[0].record(st)
        rm.encode_frag_real_batch(a8, norms, re, d_words, 0, sa)
        enc_ev[1].record(st)
        eng.search(a8, nq, sa, d_val, d_loc)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(st)
    gemm_ms, merge_ms, enc_ms = [], [], []
    for _ in range(args.steps):
        step()
        g, m_, splits = eng.kernel_ms()
        gemm_ms.append(g)
        merge_ms.append(m_)
        enc_ms.append(enc_ev[0].elapsed_time(enc_ev[1]))
    ev1.record(st)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    rm.lib()
    from rotormap._lib import check, lib
    check(lib().r2m_check_device_error(None))
    frac = mapped_fraction(d_loc.cpu().numpy(), starts0, idx.starts)
    fp64 = None
    if rank == 0 and args.fp64_sample > 0:
        g_dev = torch.from_numpy(pack.words.view(np.int32)).to(dev)
        fp64 = fp64_check(re, idx, g_dev, d_words.view(nq, re.words), d_loc, d_val, args.fp64_sample, 13)
        del g_dev

    # the read encoder alone: L2 flushed (a 256 MiB write) before each launch,
    # CUDA events around the launch only, outside the timed region
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    enc_alone = []
    for i in range(12):
        flush.fill_(i & 0xFF)
        enc_ev[0].record(st)
        rm.encode_frag_real_batch(a8, norms, re, d_words, 0, sa)
        enc_ev[1].record(st)
        enc_ev[1].synchronize()
        if i >= 2:
            enc_alone.append(enc_ev[0].elapsed_time(enc_ev[1]))
    del flush

    # end to end through the public API with host buffers
    mapper = rm.Mapper(eng, re)
    mapper.h_words[:nq].numpy().view(np.uint32)[:] = words
    for _ in range(2):
        mapper.map_words(nb=nq)
    e2e_t = []
    for _ in range(args.steps):
        t1 = time.perf_counter()
        mapper.map_words(nb=nq)
        e2e_t.append(time.perf_counter() - t1)
    e2e_s = sum(e2e_t) / len(e2e_t)

    if world > 1:
        from rotormap.dist import max_over_ranks
        ms, e2e_s = max_over_ranks([ms, e2e_s], device=dev)

    if rank == 0:
        pk, basis = peaks()
        peak = 2.0 * pk["bf16_tflops_sustained"]
        g_avg = sum(gemm_ms) / len(gemm_ms)
        flops = 2.0 * nq * N * re.rdim
        achieved = flops / (g_avg * 1e-3) / 1e12
        enc_bytes = nq * (re.words * 4 + re.rdim + 4 + 4 * M)
        # tensor-pipe estimate from the clock: the dense fp8 rate of an SM's
        # tensor pipe, 16,384 FLOP per clock (x 148 SMs x ~1.86 GHz = the
        # nominal 4.5 PFLOP/s), times the SMs and the sampled median clock
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        pipe_peak = 16384.0 * sms * (clk["sm_mhz"] or 0) * 1e6 / 1e12 if clk.get("sm_mhz") else None
        line = {
            "metric": METRIC, "value": nq * world / (ms * 1e-3), "unit": "reads/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "e4m3 (fp32 accumulate, per-row fp32 scales)",
            "data": "synthetic",
            "config": {"workload": f"kernel microbench: Q={nq} x {K_BASES}bp reads (5% subs) vs N={N} index "
                                   f"columns (k={K_BASES}, kstep={KSTEP}, fwd+rc), s{S} m{M} c{C} rdim {re.rdim}, "
                                   f"top-{TOPK}, scaled e4m3",
                       "reads_per_gpu": nq, "index_cols": N, "k": TOPK, "splits": splits,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs > L2 (34 GB index streamed every step)"},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak,
                         "traffic": SMALL_CASE_DRAM_BYTES * N / SMALL_CASE_COLS if nq == Q else None,
                         "traffic_algorithmic": nq * re.rdim + N * re.rdim,
                         "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum of one launch of "
                                         "65,536 reads x 2,097,152 columns (ncu, a 4.3 GB index) scaled by "
                                         "the column count: the index is read once per wave of paced CTA "
                                         "pairs, ~4x its size",
                         "kernel": ("k_gemm_topk2 (CTA-pair tcgen05 fp8 GEMM + fused top-20)" if nq > 128 else
                                    "k_gemm_topk (single-CTA tcgen05 fp8 GEMM + fused top-20)"),
                         "peak_basis": f"dense fp8 = 2 x {basis} sustained bf16 "
                                       f"({pk['bf16_tflops_sustained']} TFLOP/s)",
                         "tensor_pipe": {"est_active_frac": achieved / pipe_peak if pipe_peak else None,
                                         "basis": "achieved / (16384 dense fp8 FLOP per SM per clock x SMs x "
                                                  "median sampled SM clock)",
                                         "sm_mhz": clk.get("sm_mhz")},
                         "tflops_per_w": achieved / clk["power_w"] if clk.get("power_w") else None},
            "encoder": {"ms": sum(enc_ms) / len(enc_ms),
                        "achieved_gbs": enc_bytes / (sum(enc_ms) / len(enc_ms) * 1e-3) / 1e9,
                        "peak_gbs": pk["hbm_gbs"],
                        "note": "ms / achieved_gbs: in the timed step, launched after the host read the "
                                "previous step's kernel times (the GPU idles for that gap, and a sub-ms "
                                "kernel after an idle gap runs partly below the clock it had); alone_*: "
                                "10 launches after the timed region, each right behind an L2 flush",
                        "alone_ms": sum(enc_alone) / len(enc_alone),
                        "alone_gbs": enc_bytes / (sum(enc_alone) / len(enc_alone) * 1e-3) / 1e9},
            "kernels_ms": {"gemm_topk": g_avg, "merge": sum(merge_ms) / len(merge_ms),
                           "encode": sum(enc_ms) / len(enc_ms)},
            "index_build_s": t_index,
            "mapped_frac_top20": frac,
            "fp64_check": fp64,
            "e2e": {"value": nq * world / e2e_s, "unit": "reads/s", "h2d_bytes_per_step": mapper.h2d_bytes(nq),
                    "d2h_bytes_per_step": mapper.d2h_bytes(nq)},
            "gpu_launches": 3 * args.steps,
            "clocks": clk,
        }
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline(genome, words, os.cpu_count() or 1)
    eng.close()
    del idx, eng, a8, sa, d_words, mapper
    torch.cuda.empty_cache()
    if rank == 0:
        if world == 1 and not args.no_serving:
            line["serving"] = serving_leg(dev, args.requests, fp64_sample=args.fp64_sample,
                                          kernel_tflops=line["roofline"]["achieved"] if "roofline" in line else None,
                                          rows=args.serving_rows)
        if world == 1 and not args.no_precision:
            line["precision"] = precision_leg(dev, args.precision_reads, args.precision_sample)
        if world == 1 and not args.no_batching:
            line["batching"] = batching_leg(dev, args.batching_requests)
        if world == 1 and not args.no_fasta:
            line["fasta_reader"] = fasta_leg(dev)
        if world == 1 and not args.no_compact:
            line["compact"] = compact_leg(dev)
        if world == 1 and not args.no_map:
            line["run_map"] = map_leg(dev)
        if world == 1 and not args.no_gemm_bar:
            line["gemm_bar"] = gemm_bar_leg(dev)
        line["summary"] = summary(line)  # last key: the tail of the printed line
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
