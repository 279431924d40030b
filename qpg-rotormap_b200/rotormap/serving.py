"""Serving form: a continuous-batching request loop over the resident index.

The loop itself is native (r2m_server_*, csrc/server.cpp): requests
(packed read words of any count, or FASTA bytes) arrive at any time via
submit(); the library's loop thread keeps the index and every admitted
request's state resident on the device (its words and result lists), admits
requests in arrival order while their state fits both the byte budget and
the device memory free at that moment, and forms each GPU batch from
segments of all admitted requests -- a request that arrives while others are
running joins the next batch instead of waiting for them to finish.
Uploads and downloads run on a copy stream and overlap the fused search on
the compute stream.  Every read's result is independent of the batch it
lands in (the encoder and the fused top-k are deterministic per row and the
top-k order is total), so a request maps to the same result alone and in
the mix.  Requests can be cancelled, queued or in flight.

This module is the Python client: MappingServer marshals buffers (page-
locked, so the loop copies them asynchronously) and maps the loop's states
to results and exceptions.

The plain batch path (`plain_map`) is the reference contract for
comparison: one request at a time, fixed batches, synchronous per batch
(RotorMap/search/engine_fp8.jl:498-547 topk_flow).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from ._lib import R2MError, R2M_ENOMEM, check, lib
from .encoder import RopeEncoder, encode_frag_real_batch

QUEUED, ACTIVE, DONE, CANCELLED, FAILED = 0, 1, 2, 3, 4


class CancelledError(RuntimeError):
    pass


class ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("batches", "rows", "max_rows", "requests_done",
                                              "requests_cancelled", "requests_failed", "in_use_bytes",
                                              "peak_in_use_bytes", "queued", "active")]


class Request:
    """A submitted request: result() waits for it (CLOCK_MONOTONIC times,
    the clock of time.perf_counter on Linux)."""

    def __init__(self, srv, rid: int, n: int, k: int, vals=None, locs=None, words=None, fasta: bool = False):
        self._srv, self.rid, self.n, self.k = srv, rid, n, k
        self._vals, self._locs, self._words = vals, locs, words  # pinned buffers the loop writes / reads
        self.fasta = fasta
        self._out = None

    def _times(self):
        st, n = ctypes.c_int(), ctypes.c_int64()
        ta, tad, td = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(lib().r2m_server_request(self._srv._h, self.rid, ctypes.byref(st), ctypes.byref(n),
                                       ctypes.byref(ta), ctypes.byref(tad), ctypes.byref(td)))
        return st.value, ta.value, tad.value, td.value

    @property
    def state(self) -> int:
        return self._times()[0]

    @property
    def t_arrival(self) -> float:
        return self._times()[1]

    @property
    def t_admit(self) -> float:
        return self._times()[2]

    @property
    def t_done(self) -> float:
        return self._times()[3]

    @property
    def latency(self) -> float:
        _, ta, _, td = self._times()
        return td - ta

    def cancel(self) -> None:
        check(lib().r2m_server_cancel(self._srv._h, self.rid))

    def result(self, timeout: float | None = None):
        if self._out is not None:
            return self._out
        st = ctypes.c_int()
        rc = lib().r2m_server_wait(self._srv._h, self.rid, -1.0 if timeout is None else float(timeout),
                                   ctypes.byref(st))
        if rc != 0:
            if st.value in (QUEUED, ACTIVE):
                raise TimeoutError(f"request {self.rid} not done")
            check(rc)
        self._srv._live.pop(self.rid, None)  # finished: the loop no longer touches its buffers
        if st.value == CANCELLED:
            raise CancelledError(f"request {self.rid} was cancelled")
        if st.value == FAILED:
            msg = lib().r2m_server_request_error(self._srv._h, self.rid)
            raise RuntimeError(msg.decode() if msg else "request failed")
        if self.fasta:
            v = np.empty((self.n, self.k), np.float32)
            l = np.empty((self.n, self.k), np.int32)
            check(lib().r2m_server_copy_result(self._srv._h, self.rid, v.ctypes.data, l.ctypes.data))
            self._out = (v, l)
        else:
            self._out = (self._vals.numpy(), self._locs.numpy())
        return self._out

    def headers(self) -> list:
        """The parsed reads' headers of a FASTA request."""
        h = lib().r2m_server_reads(self._srv._h, self.rid)
        if not h:
            return []
        tot = ctypes.c_size_t()
        p = lib().r2m_reads_header_blob(h, ctypes.byref(tot))
        return ctypes.string_at(p, tot.value).decode("latin-1").split("\n")[:self.n]


class MappingServer:
    """Continuous-batching mapper over a fused TopKEngine (native loop)."""

    def __init__(self, eng, re: RopeEncoder, hbm_budget: int | None = None, normalize: int = 0,
                 max_queued_batches: int = 2, hbm_reserve: int = 1 << 30):
        self.eng, self.re, self.normalize = eng, re, normalize
        self.dev = eng.device
        self.k = eng.k
        self.cap = eng.rows_cap
        h = ctypes.c_void_p()
        with torch.cuda.device(self.dev):
            check(lib().r2m_server_create(eng._h, re.k, re.s, re.m, re.c, normalize,
                                          int(hbm_budget) if hbm_budget else 0, int(hbm_reserve),
                                          int(max_queued_batches), ctypes.byref(h)))
        self._h = h
        self.budget = int(hbm_budget) if hbm_budget else 0
        self._live: dict = {}

    # ------------------------------------------------------------ client API

    def request_bytes(self, n: int) -> int:
        return int(lib().r2m_server_request_bytes(self._h, n))

    def submit(self, words: np.ndarray, heads=None, t_arrival: float | None = None) -> Request:
        words = np.ascontiguousarray(words, dtype=np.uint32)
        if words.ndim != 2 or words.shape[1] != self.re.words:
            raise ValueError(f"words must be (n, {self.re.words}) uint32")
        n = words.shape[0]
        hw = torch.from_numpy(words.reshape(-1).view(np.int32)).pin_memory()
        hv = torch.empty((n, self.k), dtype=torch.float32, pin_memory=True)
        hl = torch.empty((n, self.k), dtype=torch.int32, pin_memory=True)
        rid = ctypes.c_int64()
        rc = lib().r2m_server_submit(self._h, hw.data_ptr() if n else None, n, hv.data_ptr() if n else None,
                                     hl.data_ptr() if n else None, float(t_arrival or 0.0), ctypes.byref(rid))
        if rc == R2M_ENOMEM:
            raise MemoryError(lib().r2m_last_error().decode())
        check(rc)
        r = Request(self, rid.value, n, self.k, hv, hl, hw)
        r.heads = heads
        self._live[r.rid] = r  # the loop reads and writes its buffers until it finishes
        return r

    def submit_fasta(self, data: bytes, t_arrival: float | None = None, nthreads: int = 4) -> Request:
        rid, n = ctypes.c_int64(), ctypes.c_int64()
        check(lib().r2m_server_submit_fasta(self._h, data, len(data), nthreads, float(t_arrival or 0.0),
                                            ctypes.byref(rid), ctypes.byref(n)))
        return Request(self, rid.value, n.value, self.k, fasta=True)

    def stats(self) -> ServerStats:
        st = ServerStats()
        check(lib().r2m_server_get_stats(self._h, ctypes.byref(st)))
        return st

    @property
    def batches(self) -> int:
        return self.stats().batches

    @property
    def in_use(self) -> int:
        return self.stats().in_use_bytes

    def close(self, wait: bool = True):
        if self._h:
            h, self._h = self._h, None
            try:
                check(lib().r2m_server_destroy(h, 0 if wait else 1))
            finally:
                self._live.clear()  # the loop has stopped: buffers are free to go

    def drain(self, timeout: float = 600.0):
        """Block until every submitted request has finished."""
        t0 = time.perf_counter()
        while True:
            st = self.stats()
            if st.queued == 0 and st.active == 0:
                return
            if time.perf_counter() - t0 > timeout:
                raise TimeoutError("serving loop did not drain")
            time.sleep(0.001)

    def __del__(self):
        try:
            self.close(wait=False)
        except Exception:
            pass


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
