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
around the built-in heuristic and the persistent CTA count -- on the real
shape and keeps the fastest per (bucket, N, rdim, k).
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import torch

from .encoder import RopeEncoder, encode_frag_real_batch


def bucket_rows(n: int) -> int:
    return max(128, (n + 127) // 128 * 128)


class Autotuner:
    """Picks (splits, ctas, epilogue) for an engine and row count by timing
    candidates.  The epilogue form (4 or 8 warps) depends on how
    long a work unit is, so it is only tuned when the candidates run on the
    engine itself; on a proxy index the automatic rule stays."""

    def __init__(self, cache_path: str | None = None, reps: int = 2, proxy_cols: int = 0):
        self.reps = reps
        # >0: time candidates on an engine over the first proxy_cols index
        # columns (the schedule's wave behaviour depends on read tiles x splits
        # vs CTAs, not on the column count), then apply the winner
        self.proxy_cols = proxy_cols
        self.cache: dict = {}
        self.path = Path(cache_path) if cache_path else None
        if self.path and self.path.exists():
            self.cache = json.loads(self.path.read_text())
        self.log: list = []

    @staticmethod
    def candidates(rows: int, n_cols: int, sms: int):
        m_tiles = (rows + 127) // 128
        n_tiles = (n_cols + 255) // 256
        smin = max(1, math.ceil(4 * sms / m_tiles))
        cand = {0}
        for s in (smin, 2 * smin, max(1, smin // 2), math.ceil(sms / m_tiles), math.ceil(2 * sms / m_tiles),
                  math.ceil(8 * sms / m_tiles)):
            if 1 <= s <= min(128, n_tiles):
                cand.add(int(s))
        out = [(s, 0) for s in sorted(cand)]
        out.append((0, sms - 4 if sms > 8 else sms))
        return out

    def key(self, eng, rows: int) -> str:
        return f"{rows}:{eng.N}:{eng.rdim}:{eng.k}:{eng.score}"

    def tune(self, eng, A8: torch.Tensor, rows: int, scaleA=None, stream=None):
        k = self.key(eng, rows)
        if k in self.cache:
            s, c, *rest = self.cache[k]
            ep = rest[0] if rest else "auto"
            eng.set_tuning(s, c, epilogue=ep)
            return s, c
        sms = torch.cuda.get_device_properties(eng.device).multi_processor_count
        st = stream or torch.cuda.current_stream(eng.device)
        target = eng
        if 0 < self.proxy_cols < eng.N:
            from .engine import TopKEngine
            sb = eng.scaleB[:self.proxy_cols] if eng.scaleB is not None else None
            target = TopKEngine(eng.B[:self.proxy_cols], k=eng.k, rows_cap=eng.rows_cap, score=eng.score, scaleB=sb)
        def timed(s, c, ep):
            target.set_tuning(s, c, epilogue=ep)
            target.search(A8, rows, scaleA, stream=st)  # warm
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(self.reps):
                target.search(A8, rows, scaleA, stream=st)
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / self.reps
            self.log.append({"rows": rows, "splits": s, "ctas": c, "epilogue": ep, "ms": ms})
            return ms

        best, best_ms = (0, 0, "auto"), float("inf")
        for s, c in self.candidates(rows, eng.N, sms):
            ms = timed(s, c, "auto")
            if ms < best_ms:
                best, best_ms = (s, c, "auto"), ms
        if target is eng and eng.k <= 32:  # the fused kernels' two epilogue forms
            for ep in ("4", "8"):
                ms = timed(best[0], best[1], ep)
                if ms < best_ms:
                    best, best_ms = (best[0], best[1], ep), ms
        if target is not eng:
            target.close()
        eng.set_tuning(best[0], best[1], epilogue=best[2])
        self.cache[k] = list(best)
        if self.path:
            self.path.write_text(json.dumps(self.cache))
        return best[0], best[1]


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
            self._step(rows)  # eager warm-up (first calls set kernel attributes)
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
