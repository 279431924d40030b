"""The allocation-free search entry point (r2m_batch_gemm_topk_noalloc).

It serves callers that cannot allocate device memory while they map reads
(latency-bound serving loops, where a cudaMalloc would synchronize the
device, and hosts whose memory pool owns the device memory).  It runs the
engine's automatic schedule, so its results must equal the engine path's
(r2m_batch_gemm_topk) on the same inputs bit for bit, call after call: the
shared scratch keeps the previous call's contents, which must not leak into
the next.  On integer-valued e4m3 data (every fp32 sum exact) the results
must also equal the oracle's brute force, ties included.
This file is collected last so a failure here comes after every other test.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as orc

import rotormap as rm
from rotormap._lib import R2M_ETIMEOUT, R2MError, check, lib, ptr

pytestmark = pytest.mark.gpu

E4M3_INT = np.array([0xC4, 0xC0, 0xB8, 0x00, 0x38, 0x40, 0x44], np.uint8)  # -3..3


def _noalloc(B, sb, A, sa, nb, k, mode):
    v = torch.full((nb, k), 7.0, dtype=torch.float32, device="cuda")
    l = torch.full((nb, k), 7, dtype=torch.int32, device="cuda")
    check(lib().r2m_batch_gemm_topk_noalloc(ptr(B), ptr(sb), B.shape[1], B.shape[0], ptr(A), ptr(sa), nb, k,
                                            mode, ptr(v), ptr(l), torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return v.cpu().numpy(), l.cpu().numpy()


def _engine(B, sb, A, sa, nb, k, score, kernel="auto"):
    eng = rm.TopKEngine(B, k=k, rows_cap=nb, score=score, scaleB=sb, kernel=kernel)
    v, l = eng.search(A, nb, sa)
    torch.cuda.synchronize()
    eng.close()
    return v.cpu().numpy(), l.cpu().numpy()


@pytest.mark.parametrize("nbs", [(1000, 300), (100, 37)])
def test_noalloc_matches_engine_and_oracle_twice_in_a_row(nbs):
    """A taller call, then a shorter one over the same scratch; CTA-pair
    kernel (nb > 128) and single-CTA kernel (nb <= 128)."""
    rng = np.random.default_rng(77)
    # exact integer scores: results must be identical, ties included
    Bh = E4M3_INT[rng.integers(0, 7, size=(30000, 256))]
    B = torch.from_numpy(Bh).cuda()
    for nb in nbs:
        Ah = E4M3_INT[rng.integers(0, 7, size=(nb, 256))]
        A = torch.from_numpy(Ah).cuda()
        ev, el = _engine(B, None, A, None, nb, 20, "f16")
        nv, nl = _noalloc(B, None, A, None, nb, 20, 0)
        assert np.array_equal(nv, ev) and np.array_equal(nl, el)
        ov, ol = orc.topk_e4m3(Ah, Bh, 20, 0)
        assert np.array_equal(nv, ov) and np.array_equal(nl, ol)


def test_noalloc_scaled_realistic_twice():
    rng = np.random.default_rng(5)
    B = torch.from_numpy(E4M3_INT[rng.integers(0, 7, size=(20000, 2048))]).cuda()
    sb = torch.from_numpy(rng.uniform(0.5, 2.0, 20000).astype(np.float32)).cuda()
    A = torch.from_numpy(E4M3_INT[rng.integers(0, 7, size=(513, 2048))]).cuda()
    sa = torch.from_numpy(rng.uniform(0.5, 2.0, 513).astype(np.float32)).cuda()
    ev, el = _engine(B, sb, A, sa, 513, 20, "scaled")
    for _ in range(2):
        nv, nl = _noalloc(B, sb, A, sa, 513, 20, 2)
        # same kernel (CTA pairs at 513 reads), same splits, same epilogue
        # form as the automatic engine: identical results
        assert np.array_equal(nv, ev) and np.array_equal(nl, el)
    # the single-CTA kernel of a forced engine differs only in per-column
    # accumulation order: scores within fp32 rounding, same locations
    sv, sl = _engine(B, sb, A, sa, 513, 20, "scaled", kernel="1sm")
    np.testing.assert_allclose(nv, sv, rtol=0, atol=2e-5)
    assert np.array_equal(nl, sl)


def test_noalloc_rejects_oversized_batch():
    B = torch.zeros((1000, 64), dtype=torch.uint8, device="cuda")
    nb = 300_000
    A = torch.zeros((nb, 64), dtype=torch.uint8, device="cuda")
    v = torch.empty((nb, 20), dtype=torch.float32, device="cuda")
    l = torch.empty((nb, 20), dtype=torch.int32, device="cuda")
    with pytest.raises(R2MError, match="allocation-free scratch"):
        check(lib().r2m_batch_gemm_topk_noalloc(ptr(B), None, 64, 1000, ptr(A), None, nb, 20, 0, ptr(v),
                                                ptr(l), None))


def test_noalloc_timeout_marks_rows_and_context_stays_usable():
    """The give-up handling without a fault: a bounded wait on an mbarrier
    nothing arrives on runs out (~1 ms), every row becomes NaN / -1, the
    table writer names the timeout, the engine path's error word is not
    touched, and the next search on the same context is exact."""
    nb, k = 50, 20
    v = torch.zeros((nb, k), dtype=torch.float32, device="cuda")
    l = torch.zeros((nb, k), dtype=torch.int32, device="cuda")
    check(lib().r2m_selftest_noalloc_timeout(2_000_000, nb, k, ptr(v), ptr(l), None))
    torch.cuda.synchronize()
    assert torch.isnan(v).all() and (l == -1).all()
    assert lib().r2m_check_device_error(None) == 0
    # the match-table writer refuses such rows with a timeout
    vals, locs = v.cpu().numpy(), l.cpu().numpy()
    heads = b"".join(b">r%d\n" % i for i in range(nb))
    strand = np.zeros(4, np.uint8)
    starts = np.ones(4, np.int64)
    col_rec = np.zeros(4, np.int32)
    out = ctypes.c_void_p()
    rc = lib().r2m_format_table(vals.ctypes.data, locs.ctypes.data, nb, k, heads, len(heads), strand.ctypes.data,
                                starts.ctypes.data, col_rec.ctypes.data, 4, b"rec\n", 4, 1, ctypes.byref(out))
    assert rc == R2M_ETIMEOUT and b"device timeout" in lib().r2m_last_error()
    # the same context maps exactly afterwards
    rng = np.random.default_rng(9)
    Bh = E4M3_INT[rng.integers(0, 7, size=(5000, 256))]
    Ah = E4M3_INT[rng.integers(0, 7, size=(300, 256))]
    nv, nl = _noalloc(torch.from_numpy(Bh).cuda(), None, torch.from_numpy(Ah).cuda(), None, 300, 20, 0)
    ov, ol = orc.topk_e4m3(Ah, Bh, 20, 0)
    assert np.array_equal(nv, ov) and np.array_equal(nl, ol)
