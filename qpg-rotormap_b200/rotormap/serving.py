"""Serving form: a continuous-batching request loop over the resident index.

Requests (packed read words of any count) arrive at any time via submit().
The loop keeps the index and every admitted request's state resident on the
device (its words, e4m3 rows and result lists), admits requests in arrival
order while their state fits the HBM budget, and forms each GPU batch from
segments of all admitted requests -- a request that arrives while others are
running joins the next batch instead of waiting for them to finish.
Request uploads and result downloads run on a copy stream and overlap the
fused search on the compute stream.  Every read's result is independent of
the batch it lands in (the encoder and the fused top-k are deterministic
per row and the top-k order is total), so a request maps to the same result
alone and in the mix.

The plain batch path (`plain_map`) is the reference contract for
comparison: one request at a time, fixed batches, synchronous per batch
(RotorMap/search/engine_fp8.jl:498-547 topk_flow).
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .encoder import RopeEncoder, encode_frag_real_batch


@dataclass
class Request:
    rid: int
    n: int
    words_h: np.ndarray
    t_arrival: float
    heads: list | None = None
    t_admit: float = 0.0
    t_done: float = 0.0
    vals: np.ndarray | None = None
    locs: np.ndarray | None = None
    error: str | None = None
    # device state
    words_d: torch.Tensor | None = None
    vals_d: torch.Tensor | None = None
    locs_d: torch.Tensor | None = None
    uploaded: torch.cuda.Event | None = None
    scheduled: int = 0
    completed: int = 0
    nbytes: int = 0
    done: threading.Event = field(default_factory=threading.Event)

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival

    def result(self, timeout: float | None = None):
        if not self.done.wait(timeout):
            raise TimeoutError(f"request {self.rid} not done")
        if self.error:
            raise RuntimeError(self.error)
        return self.vals, self.locs


class MappingServer:
    """Continuous-batching mapper over a fused TopKEngine."""

    def __init__(self, eng, re: RopeEncoder, hbm_budget: int | None = None, normalize: int = 0,
                 max_queued_batches: int = 2):
        self.eng, self.re, self.normalize = eng, re, normalize
        self.dev = eng.device
        self.k = eng.k
        self.cap = eng.rows_cap
        self.scaled = eng.score == "scaled"
        free, _ = torch.cuda.mem_get_info(self.dev)
        self.budget = hbm_budget if hbm_budget is not None else int(free * 0.5)
        self.in_use = 0
        self.comp = torch.cuda.Stream(self.dev)
        self.copy = torch.cuda.Stream(self.dev)
        self.max_queued = max_queued_batches
        # one batch slot: stream order on `comp` serialises its reuse
        self.norms = torch.empty((self.cap, re.m), dtype=torch.float32, device=self.dev)
        self.vals = torch.empty((self.cap, self.k), dtype=torch.float32, device=self.dev)
        self.locs = torch.empty((self.cap, self.k), dtype=torch.int32, device=self.dev)
        self._lock = threading.Condition()
        self._waiting: collections.deque = collections.deque()
        self._active: list = []
        self._inflight: collections.deque = collections.deque()  # (event, [(req, lo, n)])
        self._downloads: collections.deque = collections.deque()  # (event, req)
        self._next_id = 0
        self._stop = False
        self.batches = 0
        self.batch_rows = []
        self._thread = threading.Thread(target=self._loop, name="rotormap-serving", daemon=True)
        self._thread.start()

    # ------------------------------------------------------------ client API

    def request_bytes(self, n: int) -> int:
        return n * (self.re.words * 4 + self.k * 8)

    def submit(self, words: np.ndarray, heads=None, t_arrival: float | None = None) -> Request:
        words = np.ascontiguousarray(words, dtype=np.uint32)
        if words.ndim != 2 or words.shape[1] != self.re.words:
            raise ValueError(f"words must be (n, {self.re.words}) uint32")
        n = words.shape[0]
        nbytes = self.request_bytes(n)
        if nbytes > self.budget:
            raise MemoryError(f"request of {n} reads needs {nbytes} B > the HBM budget {self.budget} B")
        with self._lock:
            r = Request(self._next_id, n, words, t_arrival if t_arrival is not None else time.perf_counter(),
                        heads, nbytes=nbytes)
            self._next_id += 1
            if n == 0:
                r.vals = np.zeros((0, self.k), np.float32)
                r.locs = np.zeros((0, self.k), np.int32)
                r.t_done = time.perf_counter()
                r.done.set()
                return r
            self._waiting.append(r)
            self._lock.notify_all()
        return r

    def close(self, wait: bool = True):
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        if wait:
            self._thread.join()

    def drain(self, timeout: float = 600.0):
        """Block until every submitted request has completed."""
        t0 = time.perf_counter()
        with self._lock:
            while self._waiting or self._active or self._inflight or self._downloads:
                if time.perf_counter() - t0 > timeout:
                    raise TimeoutError("serving loop did not drain")
                self._lock.wait(0.01)

    # ------------------------------------------------------------ the loop

    def _admit(self):
        while self._waiting and self.in_use + self._waiting[0].nbytes <= self.budget:
            r = self._waiting.popleft()
            r.t_admit = time.perf_counter()
            self.in_use += r.nbytes
            with torch.cuda.stream(self.copy):
                hw = torch.from_numpy(r.words_h.reshape(-1).view(np.int32)).pin_memory()
                r.words_d = hw.to(self.dev, non_blocking=True)
                r.vals_d = torch.empty((r.n, self.k), dtype=torch.float32, device=self.dev)
                r.locs_d = torch.empty((r.n, self.k), dtype=torch.int32, device=self.dev)
                r.uploaded = torch.cuda.Event()
                r.uploaded.record(self.copy)
            r._pinned = hw  # keep the staging alive until the copy ran
            self._active.append(r)

    def _launch_batch(self):
        segs, off = [], 0
        for r in self._active:
            if off >= self.cap:
                break
            left = r.n - r.scheduled
            if left <= 0:
                continue
            take = min(left, self.cap - off)
            segs.append((r, r.scheduled, take, off))
            r.scheduled += take
            off += take
        if not segs:
            return False
        nb = off
        eng, W = self.eng, self.re.words
        with torch.cuda.stream(self.comp):
            for r, lo, n, o in segs:
                self.comp.wait_event(r.uploaded)
                sa = eng.scaleA[o:o + n] if self.scaled else None
                encode_frag_real_batch(eng.a8[o:o + n], self.norms[o:o + n], self.re,
                                       r.words_d[lo * W:(lo + n) * W], self.normalize, sa, self.comp)
            eng.search(eng.a8[:nb], nb, eng.scaleA[:nb] if self.scaled else None, self.vals[:nb],
                       self.locs[:nb], self.comp)
            for r, lo, n, o in segs:
                r.vals_d[lo:lo + n].copy_(self.vals[o:o + n], non_blocking=True)
                r.locs_d[lo:lo + n].copy_(self.locs[o:o + n], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.comp)
        self._inflight.append((ev, [(r, lo, n) for r, lo, n, _ in segs]))
        self.batches += 1
        self.batch_rows.append(nb)
        return True

    def _retire(self):
        progressed = False
        while self._inflight and self._inflight[0][0].query():
            _, segs = self._inflight.popleft()
            progressed = True
            for r, lo, n in segs:
                r.completed += n
                if r.completed == r.n:
                    with torch.cuda.stream(self.copy):
                        r.vals = torch.empty((r.n, self.k), dtype=torch.float32, pin_memory=True)
                        r.locs = torch.empty((r.n, self.k), dtype=torch.int32, pin_memory=True)
                        r.vals.copy_(r.vals_d, non_blocking=True)
                        r.locs.copy_(r.locs_d, non_blocking=True)
                        ev = torch.cuda.Event()
                        ev.record(self.copy)
                    self._downloads.append((ev, r))
            self._active = [r for r in self._active if r.completed < r.n]
        while self._downloads and self._downloads[0][0].query():
            _, r = self._downloads.popleft()
            r.t_done = time.perf_counter()
            r.vals, r.locs = r.vals.numpy(), r.locs.numpy()
            self.in_use -= r.nbytes
            r.words_d = r.vals_d = r.locs_d = None
            r._pinned = None
            r.done.set()
            progressed = True
        return progressed

    def _loop(self):
        torch.cuda.set_device(self.dev)
        while True:
            with self._lock:
                if self._stop and not (self._waiting or self._active or self._inflight or self._downloads):
                    return
                try:
                    progressed = self._retire()
                    self._admit()
                    launched = False
                    if len(self._inflight) < self.max_queued:
                        launched = self._launch_batch()
                except Exception as e:  # fail every pending request, keep the loop alive
                    for r in list(self._waiting) + self._active:
                        r.error = f"{type(e).__name__}: {e}"
                        r.done.set()
                    self._waiting.clear()
                    self._active.clear()
                    progressed, launched = True, False
                if not (progressed or launched):
                    self._lock.wait(0.0005)
                else:
                    self._lock.notify_all()


def plain_map(eng, re: RopeEncoder, requests, batch: int = 8192, normalize: int = 0, clock=None):
    """The plain batch path over a request list, in arrival order, one request
    at a time, fixed batches, synchronous per batch -> per-request (vals, locs)
    and completion times.  `requests`: [(t_arrival, words)]; `clock` waits
    until each arrival time (wall-clock replay)."""
    dev = eng.device
    st = torch.cuda.Stream(dev)
    out = []
    W = re.words
    norms = torch.empty((batch, re.m), dtype=torch.float32, device=dev)
    dv = torch.empty((batch, eng.k), dtype=torch.float32, device=dev)
    dl = torch.empty((batch, eng.k), dtype=torch.int32, device=dev)
    scaled = eng.score == "scaled"
    for t_arr, words in requests:
        if clock is not None:
            clock(t_arr)
        n = words.shape[0]
        vals = np.empty((n, eng.k), np.float32)
        locs = np.empty((n, eng.k), np.int32)
        for lo in range(0, n, batch):
            nb = min(batch, n - lo)
            hw = torch.from_numpy(np.ascontiguousarray(words[lo:lo + nb]).reshape(-1).view(np.int32)).pin_memory()
            with torch.cuda.stream(st):
                dw = hw.to(dev, non_blocking=True)
                sa = eng.scaleA[:nb] if scaled else None
                encode_frag_real_batch(eng.a8[:nb], norms[:nb], re, dw, normalize, sa, st)
                eng.search(eng.a8, nb, sa, dv[:nb], dl[:nb], st)
                v = dv[:nb].to("cpu", non_blocking=True)
                l = dl[:nb].to("cpu", non_blocking=True)
            st.synchronize()
            vals[lo:lo + nb] = v.numpy()
            locs[lo:lo + nb] = l.numpy()
        out.append((time.perf_counter(), vals, locs))
    return out
