"""The plain batch path (the reference engine's structure on the B200:
cuBLASLt fp8 GEMM into fp16 chunks + segmented top-k) against the oracle's
restatement of the reference's chunk loop and tie rules, and against the
fused engine."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from topk_check import assert_topk_rows, oracle_scores_at

import rotormap as rm

pytestmark = pytest.mark.gpu

E4M3_INT = np.array([0xC4, 0xC0, 0xB8, 0x00, 0x38, 0x40, 0x44], np.uint8)  # -3..3


def _plain(A8, B8, nb, w):
    B = torch.from_numpy(B8).cuda()
    eng = rm.PlainEngine(B, k=20, w=w, rows_cap=nb)
    eng.a8[:nb] = torch.from_numpy(A8).cuda()
    v, l = eng.search(eng.a8, nb)
    torch.cuda.synchronize()
    eng.close()
    return v.cpu().numpy(), l.cpu().numpy()


@pytest.mark.parametrize("nb,N,w", [(64, 100, 37), (33, 2048, 512), (100, 3000, 3000), (40, 25, 25),
                                    (16, 20, 20), (70, 5000, 1024)])
def test_plain_path_matches_reference_chunk_loop_exactly(nb, N, w):
    """Integer-valued operands: fp32 sums and fp16 storage are exact, so the
    plain path must reproduce the reference algorithm bit for bit,
    including which of several tied columns it keeps."""
    rng = np.random.default_rng(nb + N)
    A8 = E4M3_INT[rng.integers(0, 7, size=(nb, 64))]
    B8 = E4M3_INT[rng.integers(0, 7, size=(N, 64))]
    v, l = _plain(A8, B8, nb, w)
    t = orc.e4m3_table()
    scores = (t[A8].astype(np.float64) @ t[B8].astype(np.float64).T).astype(np.float32)
    dv, dl = orc.batch_topk_ref(scores, w)
    assert np.array_equal(v, dv)
    assert np.array_equal(l, dl)


def test_plain_path_agrees_with_fused_engine_on_realistic_data():
    rng = np.random.default_rng(3)
    nb, N = 1000, 300_000
    x = rng.standard_normal((nb + N, 2048)).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    q = orc.quantize_parity(x)
    A8, B8 = q[:nb], q[nb:]
    v, l = _plain(A8, B8, nb, 65536)
    B = torch.from_numpy(B8).cuda()
    eng = rm.TopKEngine(B, k=20, rows_cap=nb, score="f16")
    fv, fl = eng.search(torch.from_numpy(A8).cuda())
    fv, fl = fv.cpu().numpy(), fl.cpu().numpy()
    # fp16 scores: the two paths may differ by one fp16 step (2^-10 near 1);
    # every location where they differ must be a tie within that step
    assert_topk_rows(v, l, fv, fl, oracle_scores_at(A8, B8, l, 0), tol=1e-3, N=N)
