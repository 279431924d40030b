"""Host-ring engine (r2m_compact_*, the CompactEngine of
RotorMap/search/engine_compact.jl:256-343): an index in host memory streamed
through a device chunk ring gives the resident engine's results bit for bit
-- values, locations and tie order -- in every score mode."""
import numpy as np
import pytest
import torch

import rotormap as rm

from test_gpu_search import int_e4m3, unit_e4m3

pytestmark = pytest.mark.gpu


def resident(A8, B8, k, score="f16", scaleA=None, scaleB=None):
    B = torch.from_numpy(B8).cuda()
    sb = torch.from_numpy(scaleB).cuda() if scaleB is not None else None
    sa = torch.from_numpy(scaleA).cuda() if scaleA is not None else None
    eng = rm.TopKEngine(B, k=k, rows_cap=A8.shape[0], score=score, scaleB=sb)
    v, l = eng.search(torch.from_numpy(A8).cuda(), A8.shape[0], sa)
    out = v.cpu().numpy(), l.cpu().numpy()
    eng.close()
    return out


def compact(A8, B8, k, score="f16", scaleA=None, scaleB=None, chunk_cols=4096, depth=3, pin=True, repeat=1):
    eng = rm.CompactEngine(B8, k=k, rows_cap=A8.shape[0], score=score, scaleB=scaleB, chunk_cols=chunk_cols,
                           depth=depth, pin=pin)
    A = torch.from_numpy(A8).cuda()
    sa = torch.from_numpy(scaleA).cuda() if scaleA is not None else None
    outs = []
    for _ in range(repeat):
        v, l = eng.search(A, A8.shape[0], sa)
        outs.append((v.cpu().numpy(), l.cpu().numpy()))
    chunks = eng.chunks
    eng.close()
    return outs, chunks


@pytest.mark.parametrize("score", ["f16", "f32"])
@pytest.mark.parametrize("nb,N,chunk", [(300, 50_000, 4096), (129, 20_000, 256), (1000, 9_000, 8192),
                                        (64, 70_001, 65_536)])
def test_ring_equals_resident_with_ties(score, nb, N, chunk):
    """Integer-valued scores (exact in every order) with many equal values,
    and exact duplicate columns placed across chunk boundaries."""
    rng = np.random.default_rng(nb + N)
    rdim = 256
    A8, _ = int_e4m3(rng, (nb, rdim), -1, 1)
    B8, _ = int_e4m3(rng, (N, rdim), -1, 1)
    for c in list(range(0, N - chunk - 7, max(chunk // 2, 1)))[:40]:
        B8[c + chunk + 3] = B8[c]  # a later chunk holds the same column
    v0, l0 = resident(A8, B8, 20, score)
    outs, chunks = compact(A8, B8, 20, score, chunk_cols=chunk, repeat=2)
    assert chunks == -(-N // chunk)
    for v, l in outs:
        assert np.array_equal(v, v0) and np.array_equal(l, l0)


def test_ring_scaled_equals_resident():
    rng = np.random.default_rng(5)
    nb, N, rdim = 257, 40_000, 256
    A8 = unit_e4m3(rng, nb, rdim)
    B8 = unit_e4m3(rng, N, rdim)
    sa = rng.uniform(0.5, 2.0, nb).astype(np.float32)
    sb = rng.uniform(0.5, 2.0, N).astype(np.float32)
    v0, l0 = resident(A8, B8, 32, "scaled", sa, sb)
    outs, _ = compact(A8, B8, 32, "scaled", sa, sb, chunk_cols=3000, depth=2, repeat=2)
    for v, l in outs:
        assert np.array_equal(v, v0) and np.array_equal(l, l0)


@pytest.mark.parametrize("pin", [True, False])
def test_ring_fixed_slots_and_pageable_host(pin):
    """chunks <= depth: every chunk keeps its slot across searches; a
    pageable host index gives the same results as a page-locked one."""
    rng = np.random.default_rng(9)
    nb, N, rdim = 200, 10_000, 128
    A8 = unit_e4m3(rng, nb, rdim)
    B8 = unit_e4m3(rng, N, rdim)
    v0, l0 = resident(A8, B8, 20)
    outs, chunks = compact(A8, B8, 20, chunk_cols=4000, depth=3, pin=pin, repeat=3)
    assert chunks == 3
    for v, l in outs:
        assert np.array_equal(v, v0) and np.array_equal(l, l0)


def test_ring_rejects_bad_arguments():
    B8 = np.zeros((1000, 128), np.uint8)
    with pytest.raises(rm.R2MError):
        rm.CompactEngine(B8, k=20, chunk_cols=100)          # chunk_cols < 256
    with pytest.raises(rm.R2MError):
        rm.CompactEngine(B8, k=20, depth=1)
    with pytest.raises(ValueError):
        rm.CompactEngine(B8, k=20, score="scaled")          # no scaleB
    eng = rm.CompactEngine(B8, k=20, rows_cap=16, chunk_cols=256)
    with pytest.raises(ValueError):
        eng.search(torch.zeros((17, 128), dtype=torch.uint8, device="cuda"))
    eng.close()


def test_compact_stream_ring_equals_resident(tmp_path):
    """rope_topk_stream_compact: the uploaded index (resident = True), the
    host ring streaming every chunk (resident_chunks = 0) and the ring
    keeping what fits (the default "auto") yield the same batches."""
    from rotormap import synth
    heads = [">c1", ">c2"]
    recs = synth.random_genome([60_000, 40_000], seed=4)
    re = rm.RopeEncoder(k=150, s=8, m=4, c=4)
    idx = rm.build_index(re, synth.genome_fasta(heads, recs), kstep=15, scaled=True)
    reads, hd, _, _ = synth.sample_reads_even(heads, recs, 300, 150, 0.05, seed=8)
    p = tmp_path / "r.fa"
    p.write_bytes(synth.reads_fasta(hd, reads))
    Bh = idx.embeds8.cpu().numpy()
    sb = idx.scales.cpu().numpy() if isinstance(idx.scales, torch.Tensor) else np.asarray(idx.scales)
    a = list(rm.rope_topk_stream_compact(re, str(p), Bh, k=20, batch_size=128, score="scaled", scaleB=sb,
                                         resident=True))
    b = list(rm.rope_topk_stream_compact(re, str(p), Bh, k=20, batch_size=128, score="scaled", scaleB=sb,
                                         resident=False, chunk_cols=2048, resident_chunks=0))
    c = list(rm.rope_topk_stream_compact(re, str(p), Bh, k=20, batch_size=128, score="scaled", scaleB=sb,
                                         resident=False, chunk_cols=2048, resident_chunks="auto"))
    assert [x.heads for x in a] == [x.heads for x in b] == [x.heads for x in c]
    for x, y, z in zip(a, b, c):
        assert np.array_equal(x.vals, y.vals) and np.array_equal(x.locs, y.locs)
        assert np.array_equal(x.vals, z.vals) and np.array_equal(x.locs, z.locs)


@pytest.mark.parametrize("nres,depth", [(1, 2), (2, 2), (3, 3), (5, 2), (9, 2), (0, 2)])
@pytest.mark.parametrize("score", ["f16", "scaled"])
def test_ring_with_resident_chunks(nres, depth, score):
    """Leading chunks kept on the device (copied once), the rest streamed
    through the ring (or given slots of their own when they are few): the
    same results as the resident engine, search after search."""
    rng = np.random.default_rng(nres * 7 + depth)
    nb, N, rdim = 160, 30_000, 128
    A8, _ = int_e4m3(rng, (nb, rdim), -1, 1)
    B8, _ = int_e4m3(rng, (N, rdim), -1, 1)
    sa = rng.uniform(0.5, 2.0, nb).astype(np.float32) if score == "scaled" else None
    sb = rng.uniform(0.5, 2.0, N).astype(np.float32) if score == "scaled" else None
    v0, l0 = resident(A8, B8, 20, score, sa, sb)
    eng = rm.CompactEngine(B8, k=20, rows_cap=nb, score=score, scaleB=sb, chunk_cols=6000, depth=depth,
                           resident_chunks=nres)
    assert eng.chunks == 5 and eng.resident_chunks == min(nres, 5)
    A = torch.from_numpy(A8).cuda()
    sat = torch.from_numpy(sa).cuda() if sa is not None else None
    for _ in range(3):
        v, l = eng.search(A, nb, sat)
        assert np.array_equal(v.cpu().numpy(), v0) and np.array_equal(l.cpu().numpy(), l0)
    eng.close()


def test_auto_resident_chunks_fit_free_memory():
    free, _ = torch.cuda.mem_get_info()
    n = rm.CompactEngine.auto_resident_chunks(10_000_000, 2048, 1 << 20, 3)
    assert 0 <= n <= 10 and (n + 3) * ((10_000_000 // 10 + 5) * 2048) <= free
