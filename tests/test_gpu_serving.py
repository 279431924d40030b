"""Serving form: continuous batching over the resident index.

Each request's result must be the same alone and in the mix (the serving
contract), requests must be admitted within the HBM budget, and the served
results must agree with the plain batch path."""
import threading
import time

import numpy as np
import pytest

import rotormap as rm
import torch
from rotormap import serving, synth
from topk_check import assert_topk_rows, oracle_scores_at

pytestmark = pytest.mark.gpu

K = 150


@pytest.fixture(scope="module")
def setup():
    heads = [">srv1 a", ">srv2 b"]
    recs = synth.random_genome([700_000, 300_000], seed=21)
    re = rm.RopeEncoder(k=K, s=8, m=4, c=4)
    idx = rm.build_index(re, synth.genome_fasta(heads, recs), kstep=15)
    rng = np.random.default_rng(4)
    sizes = [1, 7, 300, 5000, 129, 20000, 64, 12000, 2]
    reqs = []
    for i, n in enumerate(sizes):
        reads, hd, _, _ = synth.sample_reads_even(heads, recs, n, K, float(rng.uniform(0, 0.1)), seed=100 + i)
        reqs.append(synth.pack_reads(reads, K))
    return re, idx, reqs


def _encode_host(re, words):
    """The e4m3 rows the server searches with (the library's encoder)."""
    dw = torch.from_numpy(np.ascontiguousarray(words).reshape(-1).view(np.int32)).cuda()
    a8, _ = rm.encode_frag_real_batch_alloc(torch.uint8, re, dw)
    return a8.cpu().numpy()


def _serve(eng, re, reqs, budget=None, stagger=0.0):
    srv = serving.MappingServer(eng, re, hbm_budget=budget)
    handles = []
    for w in reqs:
        handles.append(srv.submit(w))
        if stagger:
            time.sleep(stagger)
    out = [h.result(timeout=300) for h in handles]
    stats = srv.stats()
    srv.close()
    return out, stats, handles


def test_each_result_same_alone_and_in_the_mix(setup):
    re, idx, reqs = setup
    eng = rm.TopKEngine(idx.embeds8, k=20, rows_cap=8192)
    mix, st, _ = _serve(eng, re, reqs, stagger=0.002)
    assert st.batches >= 5 and st.max_rows == 8192
    assert st.rows == sum(w.shape[0] for w in reqs) and st.requests_done == len(reqs)
    for w, (v, l) in zip(reqs, mix):
        (av, al), = _serve(eng, re, [w])[0]
        assert np.array_equal(v, av) and np.array_equal(l, al)
    eng.close()


def test_admission_respects_the_hbm_budget(setup):
    re, idx, reqs = setup
    eng = rm.TopKEngine(idx.embeds8, k=20, rows_cap=4096)
    srv = serving.MappingServer(eng, re)
    budget = srv.request_bytes(21000)
    srv.close()
    srv = serving.MappingServer(eng, re, hbm_budget=budget)
    hs = [srv.submit(w) for w in reqs]
    res = [h.result(timeout=300) for h in hs]
    st = srv.stats()
    assert 0 < st.peak_in_use_bytes <= budget and st.in_use_bytes == 0
    with pytest.raises(MemoryError):
        srv.submit(np.zeros((30000, re.words), np.uint32))
    srv.close()
    assert all(v.shape == (w.shape[0], 20) for w, (v, _) in zip(reqs, res))
    eng.close()


def test_admission_checks_free_device_memory_at_admission(setup):
    """With a reserve larger than the device's free memory nothing fits: a
    request with nothing ahead of it fails instead of waiting forever."""
    re, idx, reqs = setup
    eng = rm.TopKEngine(idx.embeds8, k=20, rows_cap=4096)
    free, _ = torch.cuda.mem_get_info()
    srv = serving.MappingServer(eng, re, hbm_reserve=free + (1 << 30))
    h = srv.submit(reqs[2])
    with pytest.raises(RuntimeError, match="not enough free device memory"):
        h.result(timeout=60)
    assert srv.stats().requests_failed == 1
    srv.close()
    eng.close()


def test_cancel_before_admission_and_in_flight(setup):
    """A queued request that is cancelled never runs; a request cancelled
    while its rows are on the GPU stops, and the requests around it (sharing
    its batches) still get their exact results."""
    re, idx, reqs = setup
    eng = rm.TopKEngine(idx.embeds8, k=20, rows_cap=256)  # small batches: a request spans many
    ref = [_serve(eng, re, [w])[0][0] for w in reqs]
    big = np.concatenate([reqs[5], reqs[7], reqs[5]])  # 52,000 reads: ~200 batches
    # the budget holds reqs[3] and big; reqs[2] and reqs[6] wait behind them
    srv = serving.MappingServer(eng, re, hbm_budget=srv_bytes(eng, re, reqs[3].shape[0] + big.shape[0] + 100))
    hs = [srv.submit(reqs[3]), srv.submit(big), srv.submit(reqs[2]), srv.submit(reqs[6])]
    hs[3].cancel()  # still queued (the budget holds it back)
    while hs[1].state == serving.QUEUED:
        time.sleep(0.0005)
    hs[1].cancel()  # admitted, rows in flight
    with pytest.raises(serving.CancelledError):
        hs[3].result(timeout=300)
    with pytest.raises(serving.CancelledError):
        hs[1].result(timeout=300)
    for h, want in ((hs[0], ref[3]), (hs[2], ref[2])):
        v, l = h.result(timeout=300)
        assert np.array_equal(v, want[0]) and np.array_equal(l, want[1])
    st = srv.stats()
    assert st.requests_cancelled == 2 and st.requests_done == 2
    assert st.rows < big.shape[0] + reqs[3].shape[0] + reqs[2].shape[0]  # the cancelled rows were dropped
    with pytest.raises(rm.R2MError, match="already finished"):
        hs[0].cancel()
    srv.close()
    eng.close()


def srv_bytes(eng, re, n):
    s = serving.MappingServer(eng, re)
    b = s.request_bytes(n)
    s.close()
    return b


def test_fasta_requests_and_malformed_input(setup, tmp_path):
    re, idx, reqs = setup
    heads = [">srv1 a", ">srv2 b"]
    recs = synth.random_genome([700_000, 300_000], seed=21)
    reads, hd, _, _ = synth.sample_reads_even(heads, recs, 500, K, 0.03, seed=77)
    fa = synth.reads_fasta(hd, reads)
    eng = rm.TopKEngine(idx.embeds8, k=20, rows_cap=4096)
    srv = serving.MappingServer(eng, re)
    h = srv.submit_fasta(fa)
    v, l = h.result(timeout=300)
    assert h.headers() == hd
    (wv, wl), = _serve(eng, re, [synth.pack_reads(reads, K)])[0]
    assert np.array_equal(v, wv) and np.array_equal(l, wl)
    for bad, msg in ((b"ACGT\n>r1\n" + b"A" * 200 + b"\n", "before the first"),
                     (b"", "no record"), (b"\n\n", "no record"),
                     (b">short\nACGT\n", "no record has")):
        with pytest.raises(rm.R2MError, match=msg):
            srv.submit_fasta(bad)
    srv.close()
    eng.close()


def test_bad_index_file_is_refused(tmp_path, setup):
    """A truncated reference .bin never reaches an engine or a server."""
    re, idx, reqs = setup
    p = tmp_path / "i.bin"
    idx.save(p)
    raw = p.read_bytes()
    (tmp_path / "cut.bin").write_bytes(raw[: len(raw) // 2])
    with pytest.raises(rm.R2MError, match="index .bin"):
        rm.load_index(str(tmp_path / "cut.bin"))


def test_served_results_match_plain_path(setup):
    re, idx, reqs = setup
    eng = rm.TopKEngine(idx.embeds8, k=20, rows_cap=8192)
    mix, _, _ = _serve(eng, re, reqs)
    plain = serving.plain_map(eng, re, [(0.0, w) for w in reqs], batch=8192)
    for (v, l), (_, pv, pl) in zip(mix, plain):
        assert np.array_equal(v, pv) and np.array_equal(l, pl)
    # the reference-structured engine (cuBLASLt + segmented top-k)
    peng = rm.PlainEngine(idx.embeds8, k=20, w=65536, rows_cap=8192)
    ref = serving.plain_map(peng, re, [(0.0, w) for w in reqs], batch=8192)
    # the reference-structured engine keeps an arbitrary one of tied
    # locations; every location that differs is a tie within one fp16 step
    B = idx.embeds8.cpu().numpy()
    for w, (v, l), (_, pv, pl) in zip(reqs, mix, ref):
        a8 = _encode_host(re, w)
        assert_topk_rows(v, l, pv, pl, oracle_scores_at(a8, B, l, 0), tol=1e-3, N=idx.N)
    peng.close()
    eng.close()
