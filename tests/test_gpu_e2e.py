"""End-to-end GPU checks of the mapping path on the plain-method configuration:
a 1 Mbp genome of two records (600 kbp + 400 kbp, iid ACGT), index at
s=8 m=4 c=4 with k = read length = 150 and the builder's default stride
k/10 = 15 (forward + reverse complement), reads sampled :even.

Mirrors the reference self-test floors (RotorMap/selftest.jl:190-224,
run_e2e_test in RotorMap/experiments/e2e_fp8.jl:141-163): every err = 0 read
maps with its first hit at rank 1, >= 0.90 of 5%-substitution reads map in
the top 20; and the top-k of the whole flow equals the oracle's brute force
over the same quantised operands (RotorMap/search/engine_fp8.jl:843-894)."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from topk_check import assert_topk_rows, oracle_scores_at

import rotormap as rm
from rotormap import synth

pytestmark = pytest.mark.gpu

K = 150


@pytest.fixture(scope="module")
def fixture():
    heads = [">chrA plain-method record A", ">chrB plain-method record B"]
    recs = synth.random_genome([600_000, 400_000], seed=1)
    fa = synth.genome_fasta(heads, recs)
    re = rm.RopeEncoder(k=K, s=8, m=4, c=4)
    idx = rm.build_index(re, fa, kstep=15)
    return heads, recs, re, idx


def _reads_file(tmp_path, heads, recs, n, err, seed, name, model="subs"):
    reads, hd, _, _ = synth.sample_reads_even(heads, recs, n, K, err, seed=seed, model=model)
    p = tmp_path / name
    p.write_bytes(synth.reads_fasta(hd, reads))
    return p, reads, hd


def test_index_shape(fixture):
    heads, recs, re, idx = fixture
    nwin = (600_000 - K) // 15 + 1 + (400_000 - K) // 15 + 1
    assert idx.N == 2 * nwin == 133_296
    assert idx.embeds8.shape == (133_296, 2048)


def test_selftest_err0_all_map_at_rank1(fixture, tmp_path):
    heads, recs, re, idx = fixture
    p, _, _ = _reads_file(tmp_path, heads, recs, 1000, 0.0, 42, "r0.fa")
    r = rm.map_and_count(re, str(p), idx, ktop=20, batch_size=384)
    assert r["total"] == 1000 and r["correct"] == 1000
    assert r["rank_hist"][0] == 1000
    assert r["nb"] == 3  # 1000 reads in batches of 384


def test_selftest_err5_top20_floor(fixture, tmp_path):
    heads, recs, re, idx = fixture
    p, _, _ = _reads_file(tmp_path, heads, recs, 200, 0.05, 7, "r5.fa")
    r = rm.map_and_count(re, str(p), idx, ktop=20)
    assert r["total"] == 200 and r["correct"] / 200 >= 0.90


def test_selftest_err5_floor_with_the_reference_sampler(fixture, tmp_path):
    """The self-test's mutated reads as the reference samples them: its
    edit model (substitutions, insertions, deletions) on its own Xoshiro
    draws (rotormap.jlrandom), 200 reads at err = 0.05, floor 0.90
    (RotorMap/selftest.jl:62-63, 204-222)."""
    heads, recs, re, idx = fixture
    p, _, _ = _reads_file(tmp_path, heads, recs, 200, 0.05, 11, "r5ref.fa", model="reference")
    r = rm.map_and_count(re, str(p), idx, ktop=20)
    assert r["total"] == 200 and r["correct"] / 200 >= 0.90


def test_flow_topk_equals_oracle_brute_force(fixture, tmp_path):
    """rope_topk_stream top-20 vs the oracle: reads encoded by the oracle's
    fp32 restatement and quantised like the reference, scored against the
    same stored index columns."""
    heads, recs, re, idx = fixture
    p, reads, hd = _reads_file(tmp_path, heads, recs, 300, 0.05, 9, "rq.fa")
    bats = list(rm.rope_topk_stream(re, str(p), idx.embeds8, k=20, batch_size=128))
    vals = np.concatenate([b.vals for b in bats])
    locs = np.concatenate([b.locs for b in bats])
    assert [h for b in bats for h in b.heads] == hd
    assert [b.first for b in bats] == [1, 129, 257]
    words = synth.pack_reads(reads, K)
    f32, _ = orc.rope_f32(words, K, 8, 4, 4)
    a8 = orc.quantize_parity(f32)
    B = idx.embeds8.cpu().numpy()
    ov, ol = orc.topk_e4m3(a8, B, 20, 0)
    # tolerance: one fp16 step of a score near 1 (2^-10); a location that
    # differs from the oracle's must be a tie within it (checked per entry)
    assert_topk_rows(vals, locs, ov, ol, oracle_scores_at(a8, B, locs, 0), tol=1e-3, N=idx.N)


def test_stream_device_and_host_readers_agree(fixture, tmp_path):
    """rope_topk_stream with the GPU FASTA reader and with the host reader:
    the same batches, headers, scores and locations."""
    heads, recs, re, idx = fixture
    p, _, hd = _reads_file(tmp_path, heads, recs, 300, 0.05, 13, "rd.fa")
    a = list(rm.rope_topk_stream(re, str(p), idx.embeds8, k=20, batch_size=128, reader="device"))
    b = list(rm.rope_topk_stream(re, str(p), idx.embeds8, k=20, batch_size=128, reader="host"))
    assert [x.heads for x in a] == [x.heads for x in b] and [h for x in a for h in x.heads] == hd
    for x, y in zip(a, b):
        assert x.first == y.first
        assert np.array_equal(x.vals, y.vals) and np.array_equal(x.locs, y.locs)
        assert np.array_equal(x.norms, y.norms)
    with pytest.raises(ValueError):
        next(rm.rope_topk_stream(re, str(p), idx.embeds8, reader="other"))


def test_run_map_table(fixture, tmp_path):
    heads, recs, re, idx = fixture
    p, _, hd = _reads_file(tmp_path, heads, recs, 50, 0.0, 3, "rm.fa")
    out = tmp_path / "rm.maps"
    n = rm.run_map(idx, str(p), str(out), topk=5)
    lines = out.read_text().splitlines()
    assert n == 50 and len(lines) == 250
    first = lines[0].split(" ")
    h = rm.parse_read_head(hd[0])
    assert " ".join(first[:4]) == hd[0][1:]        # header sans '>' (4 tokens)
    assert first[4] in "+-" and first[7] in ("chrA", "chrB")
    assert abs(int(first[6]) + 1 - h["start"]) < K  # 0-based window start near the read
    scores = [float(l.split(" ")[5]) for l in lines[:5]]
    assert scores == sorted(scores, reverse=True)


def test_index_save_load_map_round_trip(fixture, tmp_path):
    heads, recs, re, idx = fixture
    path = tmp_path / "g.r2mi"
    idx.save(path)
    back = rm.load_index(str(path), device="cuda")
    assert torch.equal(back.embeds8, idx.embeds8)
    p, _, _ = _reads_file(tmp_path, heads, recs, 100, 0.0, 5, "rr.fa")
    a = list(rm.rope_topk_stream(re, str(p), idx.embeds8, k=20))
    b = list(rm.rope_topk_stream(re, str(p), back.embeds8, k=20))
    assert np.array_equal(a[0].locs, b[0].locs) and np.array_equal(a[0].vals, b[0].vals)


def test_reference_bin_round_trip_maps(fixture, tmp_path):
    """The reference's index file (Julia-serialized NamedTuple, written by
    save_index): load_index memory-maps it, uploads embeds8 once and the
    search, the table and the rescoring meta match the built index."""
    heads, recs, re, idx = fixture
    path = tmp_path / "g.indexreal_fp8.bin"
    idx.save(path)
    back = rm.load_index(str(path), device="cuda")
    assert back.format == rm.FP8_FORMAT and back.N == idx.N and back.heads == idx.heads
    assert torch.equal(back.embeds8, idx.embeds8)
    assert np.array_equal(np.asarray(back.starts), idx.starts) and np.array_equal(np.asarray(back.strand), idx.strand)
    p, _, _ = _reads_file(tmp_path, heads, recs, 200, 0.05, 21, "rb.fa")
    a = list(rm.rope_topk_stream(re, str(p), idx.embeds8, k=20))
    b = list(rm.rope_topk_stream(re, str(p), back.embeds8, k=20))
    assert np.array_equal(a[0].locs, b[0].locs) and np.array_equal(a[0].vals, b[0].vals)
    # run_map straight from the .bin path (the tools/map.jl contract)
    out_a, out_b = tmp_path / "a.maps", tmp_path / "b.maps"
    rm.run_map(idx, str(p), str(out_a), topk=5)
    rm.run_map(str(path), str(p), str(out_b), topk=5)
    assert out_a.read_bytes() == out_b.read_bytes()
    # the packed genome for rescoring is rebuilt from the source FASTA
    fa = tmp_path / "g.fa"
    fa.write_bytes(synth.genome_fasta(heads, recs))
    rm.attach_genome(back, str(fa))
    assert np.array_equal(back.col_pos, idx.col_pos)


def test_row_layout_bin_quantises_like_the_reference(tmp_path):
    """An "indexreal.v1" fp16 row-layout file: index_database builds B with
    H2D + transpose + e4m3(fp32(fp16)) (index_to_f8, load.jl:75-97)."""
    rng = np.random.default_rng(12)
    N, m, c = 70_000, 1, 2
    rdim = 2 * m * 4 ** c
    rows = (rng.standard_normal((rdim, N)) * 0.3).astype(np.float16)  # Julia (N, rdim) column-major
    path = tmp_path / "rows.bin"
    rm.jlbin.write_bin(path, [("format", "indexreal.v1"), ("source", "x.fa"), ("k", 20), ("kstep", 2),
                              ("s", 3), ("m", m), ("c", c), ("normalize", 0), ("fp16", True), ("n_frag", N // 2),
                              ("embeds", rows), ("norms", np.ones((N, m), np.float32)),
                              ("heads", [">a"] * N), ("starts", np.arange(1, N + 1)),
                              ("strand", np.zeros(N, np.uint8))])
    idx = rm.load_index(str(path), device="cuda")
    want = orc.f32_to_e4m3(rows.T.astype(np.float32))
    assert np.array_equal(idx.embeds8.cpu().numpy(), want)


def test_scaled_index_maps_as_well(tmp_path):
    heads = [">s1", ">s2"]
    recs = synth.random_genome([50_000, 30_000], seed=2)
    re = rm.RopeEncoder(k=K, s=8, m=4, c=4)
    idx = rm.build_index(re, synth.genome_fasta(heads, recs), kstep=15, scaled=True)
    assert idx.scaled and idx.scales.shape == (idx.N,)
    p, _, _ = _reads_file(tmp_path, heads, recs, 200, 0.05, 8, "rs.fa")
    r = rm.map_and_count(re, str(p), idx, ktop=20)
    assert r["correct"] / r["total"] >= 0.90
