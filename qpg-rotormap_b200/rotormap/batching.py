"""Batching form: ragged request sets in one persistent launch, captured in
CUDA graphs, with schedules picked by an autotuner.

Requests of any read count share the index's fragment length k (the reader
trims every read to k, RotorMap/fasta/reader.jl:262-263), so a ragged set is
one row range: the batcher concatenates the requests' packed words into one
staging buffer, runs ONE encoder launch and ONE persistent fused GEMM/top-k
launch over all rows, and splits the result rows back per request.

The whole step (H2D of the words, encode, search, D2H of the results) is
captured once per row bucket (row count rounded up to 128 reads, the fused
kernel's read tile) into a CUDA graph and replayed; pad rows are encoded from
zero words and their results dropped.

The autotuner times the fused kernel's schedule candidates -- column splits
and persistent CTAs around the built-in heuristic, kernel, epilogue form,
pacing window and top-k reservoir size -- on the real row count and keeps
the fastest per (bucket, N, rdim, k, score).
"""
from __future__ import annotations

import json
import math
import time
from pathlib import Path

import numpy as np
import torch

from .encoder import RopeEncoder, encode_frag_real_batch


def bucket_rows(n: int) -> int:
    return max(128, (n + 127) // 128 * 128)


class Autotuner:
    """Picks the fused search's schedule for an engine and a row count by
    timing candidates on the real row count: column splits and persistent
    CTAs (around the built-in heuristic), the kernel (single CTAs or CTA
    pairs), the epilogue form (4 or 8 warps), the pair pacing window and the
    top-k reservoir size -- coordinate descent from the defaults, one knob at
    a time, each kept only when it beats the best so far by `min_gain`.

    Cost: every candidate is one warm-up and `reps` timed searches.  When
    that would exceed `budget` x the estimated time of one search of the
    real shape, candidates run on a prefix of the index columns sized to fit
    the budget, and only splits and CTAs are tuned there (the wave behaviour
    -- read tiles x splits against CTAs -- is the real one; work units are
    shorter, which misleads the other knobs).  Results are cached per (rows,
    N, rdim, k, score) and, with `cache_path` (default $R2M_TUNE_CACHE),
    kept across runs."""

    RATE = 2.5e15  # FLOP/s: a model of the fused kernel, used only to size the budget

    def __init__(self, cache_path: str | None = None, reps: int = 1, proxy_cols: int = 0,
                 budget: float = 0.15, min_proxy_tiles: int = 256, min_gain: float = 0.02):
        import os
        self.reps = reps
        self.min_gain = min_gain  # a candidate must beat the best by this fraction
        # > 0: force candidates onto the first proxy_cols index columns
        self.proxy_cols = proxy_cols
        self.budget = budget
        self.min_proxy_cols = 256 * min_proxy_tiles
        self.cache: dict = {}
        cache_path = cache_path or os.environ.get("R2M_TUNE_CACHE")
        self.path = Path(cache_path) if cache_path else None
        if self.path and self.path.exists():
            self.cache = json.loads(self.path.read_text())
        self.log: list = []
        self.last: dict = {}

    @staticmethod
    def candidates(rows: int, n_cols: int, sms: int, max_splits: int = 4):
        """(splits, ctas) candidates: the heuristic (0) and splits around it."""
        m_tiles = (rows + 127) // 128
        n_tiles = (n_cols + 255) // 256
        smin = max(1, math.ceil(4 * sms / m_tiles))
        cand = []
        for s in (smin, 2 * smin, max(1, smin // 2), math.ceil(2 * sms / m_tiles), math.ceil(8 * sms / m_tiles)):
            if 1 <= s <= min(128, n_tiles) and s not in cand:
                cand.append(int(s))
        out = [(0, 0)] + [(s, 0) for s in sorted(cand)[:max_splits]]
        if m_tiles < 4 * sms:  # few read tiles: fewer CTAs can balance the last wave
            out.append((0, sms - 4 if sms > 8 else sms))
        return out

    def key(self, eng, rows: int) -> str:
        return f"{rows}:{eng.N}:{eng.rdim}:{eng.k}:{eng.score}"

    def _proxy_cols(self, eng, rows: int, searches: int) -> int:
        if self.proxy_cols:
            return min(self.proxy_cols, eng.N)
        est = 2.0 * rows * eng.N * eng.rdim / self.RATE
        per = self.budget * est / max(searches, 1)
        cols = int(per * self.RATE / (2.0 * rows * eng.rdim))
        cols = max(cols, self.min_proxy_cols)
        return eng.N if cols >= eng.N else cols // 256 * 256

    @staticmethod
    def _apply(eng, cfg):
        eng.set_tuning(cfg["splits"], cfg["ctas"], kernel=cfg["kernel"], epilogue=cfg["epilogue"],
                       pace=cfg["pace"], kt=cfg["kt"])

    def tune(self, eng, A8: torch.Tensor, rows: int, scaleA=None, stream=None):
        k = self.key(eng, rows)
        if k in self.cache:
            cfg = self.cache[k]
            if isinstance(cfg, list):  # older cache entries: (splits, ctas[, epilogue])
                cfg = {"splits": cfg[0], "ctas": cfg[1], "kernel": "auto",
                       "epilogue": cfg[2] if len(cfg) > 2 else "auto", "pace": 0, "kt": 0}
            self._apply(eng, cfg)
            self.last = dict(cfg, cached=True)
            return cfg["splits"], cfg["ctas"]
        sms = torch.cuda.get_device_properties(eng.device).multi_processor_count
        st = stream or torch.cuda.current_stream(eng.device)
        split_c = self.candidates(rows, eng.N, sms)
        kt_c = [0] + ([32] if eng.k <= 20 else [64] if eng.k <= 32 else [])
        n_trials = len(split_c) + 1 + (2 if eng.k <= 32 else 0) + 2 + len(kt_c) - 1
        cols = self._proxy_cols(eng, rows, n_trials * (1 + self.reps))
        target = eng
        if cols < eng.N:
            from .engine import TopKEngine
            sb = eng.scaleB[:cols] if eng.scaleB is not None else None
            target = TopKEngine(eng.B[:cols], k=eng.k, rows_cap=eng.rows_cap, score=eng.score, scaleB=sb)
        t_start = time.perf_counter()

        def timed(cfg):
            self._apply(target, cfg)
            target.search(A8, rows, scaleA, stream=st)  # warm
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(self.reps):
                target.search(A8, rows, scaleA, stream=st)
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / self.reps
            self.log.append(dict(cfg, rows=rows, cols=cols, ms=ms))
            return ms

        best = {"splits": 0, "ctas": 0, "kernel": "auto", "epilogue": "auto", "pace": 0, "kt": 0}
        default_ms = best_ms = timed(best)

        def consider(**change):
            nonlocal best, best_ms
            cfg = dict(best, **change)
            if cfg == best:
                return
            ms = timed(cfg)
            if ms < best_ms * (1.0 - self.min_gain):  # noise does not move the schedule
                best, best_ms = cfg, ms

        for s, c in split_c[1:]:
            consider(splits=s, ctas=c)
        if target is eng:
            # kernel, epilogue form, pacing and reservoir size depend on how
            # long a work unit is and on how many pairs share an index tile
            # in L2 -- a column prefix changes both, so these are tuned only on
            # the real shape (on a 166K-column prefix the single-CTA kernel
            # led by 3%, on the 20M-column index it ran 27% slower)
            consider(kernel="1sm" if rows > 128 else "2sm")
            if eng.k <= 32:
                consider(epilogue="4")
                consider(epilogue="8")
            consider(pace=32)
            consider(pace=-1)
            for kt in kt_c[1:]:
                consider(kt=kt)
        if target is not eng:
            target.close()
        self._apply(eng, best)
        self.last = dict(best, ms=best_ms, default_ms=default_ms, proxy_cols=cols,
                         tune_s=time.perf_counter() - t_start, cached=False)
        self.cache[k] = best
        if self.path:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            self.path.write_text(json.dumps(self.cache))
        return best["splits"], best["ctas"]


class RaggedBatcher:
    """One launch per ragged request set, replayed from captured CUDA graphs."""

    def __init__(self, eng, re: RopeEncoder, capacity: int, normalize: int = 0, tuner: Autotuner | None = None,
                 use_graphs: bool = True):
        if capacity > eng.rows_cap:
            raise ValueError("capacity exceeds the engine rows_cap")
        self.eng, self.re, self.normalize = eng, re, normalize
        self.cap = bucket_rows(capacity)
        if self.cap > eng.rows_cap:
            raise ValueError("engine rows_cap must be a multiple of 128 at least the capacity")
        dev = eng.device
        W, k = re.words, eng.k
        self.h_words = torch.zeros((self.cap, W), dtype=torch.int32, pin_memory=True)
        self.h_vals = torch.empty((self.cap, k), dtype=torch.float32, pin_memory=True)
        self.h_locs = torch.empty((self.cap, k), dtype=torch.int32, pin_memory=True)
        self.d_words = torch.zeros((self.cap, W), dtype=torch.int32, device=dev)
        self.d_norms = torch.empty((self.cap, re.m), dtype=torch.float32, device=dev)
        self.d_vals = torch.empty((self.cap, k), dtype=torch.float32, device=dev)
        self.d_locs = torch.empty((self.cap, k), dtype=torch.int32, device=dev)
        self.stream = torch.cuda.Stream(dev)
        self.tuner = tuner
        self.use_graphs = use_graphs
        self.graphs: dict = {}
        self.launches = 0

    def _step(self, rows: int):
        eng, st = self.eng, self.stream
        sa = eng.scaleA[:rows] if eng.score == "scaled" else None
        self.d_words[:rows].copy_(self.h_words[:rows], non_blocking=True)
        encode_frag_real_batch(eng.a8[:rows], self.d_norms[:rows], self.re, self.d_words[:rows], self.normalize,
                               sa, st)
        eng.search(eng.a8[:rows], rows, sa, self.d_vals[:rows], self.d_locs[:rows], st)
        self.h_vals[:rows].copy_(self.d_vals[:rows], non_blocking=True)
        self.h_locs[:rows].copy_(self.d_locs[:rows], non_blocking=True)

    def _graph(self, rows: int):
        g = self.graphs.get(rows)
        if g is not None:
            return g
        with torch.cuda.stream(self.stream):
            if self.tuner is not None:
                sa = self.eng.scaleA[:rows] if self.eng.score == "scaled" else None
                self.tuner.tune(self.eng, self.eng.a8, rows, sa, self.stream)
            # eager warm-up on one read tile: the step's first calls load the
            # encoder and set its launch attributes outside the capture (the
            # engine loads its fused kernels when it is created)
            self._step(min(rows, 128))
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream, capture_error_mode="thread_local"):
            self._step(rows)
        self.graphs[rows] = g
        return g

    def run(self, requests):
        """Map a list of (n_i, W) uint32 word arrays -> [(vals_i, locs_i)]."""
        sizes = [int(w.shape[0]) for w in requests]
        total = sum(sizes)
        if total == 0:
            return [(np.zeros((0, self.eng.k), np.float32), np.zeros((0, self.eng.k), np.int32)) for _ in requests]
        if total > self.cap:
            raise ValueError(f"ragged set of {total} reads exceeds the capacity {self.cap}")
        rows = bucket_rows(total)
        hw = self.h_words.numpy().view(np.uint32)
        off = 0
        for w in requests:
            hw[off:off + w.shape[0]] = w
            off += w.shape[0]
        hw[off:rows] = 0
        if self.use_graphs:
            g = self._graph(rows)
            with torch.cuda.stream(self.stream):
                g.replay()
        else:
            if self.tuner is not None:
                with torch.cuda.stream(self.stream):
                    self.tuner.tune(self.eng, self.eng.a8, rows,
                                    self.eng.scaleA[:rows] if self.eng.score == "scaled" else None, self.stream)
            with torch.cuda.stream(self.stream):
                self._step(rows)
        self.stream.synchronize()
        self.launches += 1
        v, l = self.h_vals.numpy(), self.h_locs.numpy()
        out, off = [], 0
        for n in sizes:
            out.append((v[off:off + n].copy(), l[off:off + n].copy()))
            off += n
        return out
