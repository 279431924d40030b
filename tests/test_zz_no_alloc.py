"""The allocation-free search entry point (r2m_batch_gemm_topk_noalloc).

It serves callers that cannot allocate device memory while they map reads
(latency-bound serving loops, where a cudaMalloc would synchronize the
device, and hosts whose memory pool owns the device memory).  Its results must equal the engine path's
(r2m_batch_gemm_topk) on the same inputs, call after call: the shared scratch
keeps the previous call's contents, which must not leak into the next.
This file is collected last so a failure here comes after every other test.
"""

import numpy as np
import pytest
import torch

import rotormap as rm
from rotormap._lib import R2MError, check, lib, ptr

pytestmark = pytest.mark.gpu

E4M3_INT = np.array([0xC4, 0xC0, 0xB8, 0x00, 0x38, 0x40, 0x44], np.uint8)  # -3..3


def _noalloc(B, sb, A, sa, nb, k, mode):
    v = torch.full((nb, k), 7.0, dtype=torch.float32, device="cuda")
    l = torch.full((nb, k), 7, dtype=torch.int32, device="cuda")
    check(lib().r2m_batch_gemm_topk_noalloc(ptr(B), ptr(sb), B.shape[1], B.shape[0], ptr(A), ptr(sa), nb, k,
                                            mode, ptr(v), ptr(l), torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return v.cpu().numpy(), l.cpu().numpy()


def _engine(B, sb, A, sa, nb, k, score):
    eng = rm.TopKEngine(B, k=k, rows_cap=nb, score=score, scaleB=sb)
    v, l = eng.search(A, nb, sa)
    torch.cuda.synchronize()
    eng.close()
    return v.cpu().numpy(), l.cpu().numpy()


def test_noalloc_matches_engine_twice_in_a_row():
    rng = np.random.default_rng(77)
    # exact integer scores: results must be identical, ties included
    B = torch.from_numpy(E4M3_INT[rng.integers(0, 7, size=(30000, 256))]).cuda()
    A1 = torch.from_numpy(E4M3_INT[rng.integers(0, 7, size=(1000, 256))]).cuda()
    A2 = torch.from_numpy(E4M3_INT[rng.integers(0, 7, size=(300, 256))]).cuda()
    for A in (A1, A2):  # a taller call, then a shorter one over the same scratch
        nb = A.shape[0]
        ev, el = _engine(B, None, A, None, nb, 20, "f16")
        nv, nl = _noalloc(B, None, A, None, nb, 20, 0)
        assert np.array_equal(nv, ev) and np.array_equal(nl, el)


def test_noalloc_scaled_realistic_twice():
    rng = np.random.default_rng(5)
    B = torch.from_numpy(E4M3_INT[rng.integers(0, 7, size=(20000, 2048))]).cuda()
    sb = torch.from_numpy(rng.uniform(0.5, 2.0, 20000).astype(np.float32)).cuda()
    A = torch.from_numpy(E4M3_INT[rng.integers(0, 7, size=(513, 2048))]).cuda()
    sa = torch.from_numpy(rng.uniform(0.5, 2.0, 513).astype(np.float32)).cuda()
    ev, el = _engine(B, sb, A, sa, 513, 20, "scaled")
    for _ in range(2):
        nv, nl = _noalloc(B, sb, A, sa, 513, 20, 2)
        # same kernels, same per-column accumulation order: identical scores
        np.testing.assert_allclose(nv, ev, rtol=0, atol=2e-5)
        assert np.array_equal(nl, el)


def test_noalloc_rejects_oversized_batch():
    B = torch.zeros((1000, 64), dtype=torch.uint8, device="cuda")
    nb = 300_000
    A = torch.zeros((nb, 64), dtype=torch.uint8, device="cuda")
    v = torch.empty((nb, 20), dtype=torch.float32, device="cuda")
    l = torch.empty((nb, 20), dtype=torch.int32, device="cuda")
    with pytest.raises(R2MError, match="allocation-free scratch"):
        check(lib().r2m_batch_gemm_topk_noalloc(ptr(B), None, 64, 1000, ptr(A), None, nb, 20, 0, ptr(v),
                                                ptr(l), None))
