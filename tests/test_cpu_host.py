"""CPU tests of the host side: the C ABI exports, the native FASTA reader
against the oracle restatement of RotorMap/fasta/reader.jl, reference-window
enumeration (RotorMap/index/build.jl:291-324), the index container, the
map.jl table formatting and the provenance scorer.  No GPU is needed."""
import re as _re
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as orc

import rotormap as rm
from rotormap import _lib, synth
from rotormap.index import Index, batch_column_order

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    txt = (ROOT / "include" / "r2m.h").read_text()
    txt = _re.sub(r"/\*.*?\*/", "", txt, flags=_re.S)
    return sorted(set(_re.findall(r"\b(r2m_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_every_declared_symbol():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), f"{s} declared in r2m.h but not exported"
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(syms) == bound, "ctypes signatures and r2m.h disagree"
    assert L.r2m_version() >= 10000


def test_device_entry_points_fail_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(_lib.R2MError):
        _lib.require_device()


FASTA_CASES = [
    b"",
    b"no record here\nACGT\n",
    b"junk line\n>r1 first\nACGTACGTAC\nGTACGTACGT\n>r2\nAC\n",
    b">crlf\r\nACGTNNNNacgtRYK\r\nTTTT\r\n>x\r\nGGGGGGGGGGGGGGGGGGGGGG\r\n",
    b">a\nAC>GT ACGT\nAAAAAAAAAAAAAAAAAAAAA\n>b\n\n\nCCCCCCCCCCCCCCCCCCCCCCCCCCC",
    b">only header at eof",
    b">h1\nACGTACGTACGTACGTACGTACGTACGTACGT\n>h2 no newline before next\r>h3\nAAAAAAAAAAAAAAAAAAAAAAAAAAA\n",
    b">r\n" + b"ACGT" * 64 + b"\n>s\n" + b"T" * 31 + b"\n>t\n" + b"G" * 32 + b"\n>u\n" + b"C" * 33 + b"\n",
]


@pytest.mark.parametrize("k", [1, 5, 16, 17, 31, 32, 33, 150])
@pytest.mark.parametrize("ci", range(len(FASTA_CASES)))
def test_fasta_reader_matches_oracle(ci, k):
    raw = FASTA_CASES[ci]
    got = rm.fasta_reads(raw, k=k, parts=1)
    ref = orc.fasta_reads_ref(raw, k)
    assert got.heads == [h for h, _ in ref]
    if ref:
        assert np.array_equal(got.words, np.stack([w for _, w in ref]))
    else:
        assert got.words.shape[0] == 0


@pytest.mark.parametrize("seed", range(6))
def test_fasta_reader_random_layouts_match_oracle(seed):
    """Random line widths, LF/CRLF/CR line ends, lower case and non-ACGT bytes:
    the reader's 16-byte packing steps straddle every kind of line break."""
    rng = np.random.default_rng(seed)
    alphabet = np.frombuffer(b"ACGTacgtNRYn-*", np.uint8)
    out = [b"preamble\n"] if seed % 2 else []
    for r in range(40):
        n = int(rng.integers(0, 300))
        w = np.r_[[0.22] * 4, [0.02] * 4, [0.01] * 6]
        seq = alphabet[rng.choice(alphabet.size, n, p=w / w.sum() if seed % 3 else None)]
        eol = [b"\n", b"\r\n", b"\r"][int(rng.integers(0, 3))] if seed >= 3 else b"\n"
        width = int(rng.integers(1, 90))
        body = eol.join(seq[i:i + width].tobytes() for i in range(0, n, width))
        hdr_eol = b"\r\n" if eol == b"\r\n" else b"\n"
        out.append(b">rec%d %d" % (r, n) + hdr_eol + body + eol)
    raw = b"".join(out)
    for k in (1, 15, 16, 17, 48, 150):
        got = rm.fasta_reads(raw, k=k, parts=1)
        ref = orc.fasta_reads_ref(raw, k)
        assert got.heads == [h for h, _ in ref]
        if ref:
            assert np.array_equal(got.words, np.stack([w for _, w in ref]))


def test_fasta_reader_threads_do_not_change_the_result():
    recs = synth.random_genome([1000] * 6000, seed=9)
    heads = [f">rec_{i} x" for i in range(6000)]
    raw = synth.genome_fasta(heads, recs, width=60)
    assert len(raw) > (1 << 22)
    a = rm.fasta_reads(raw, k=150, parts=1)
    b = rm.fasta_reads(raw, k=150, parts=8)
    assert a.heads == b.heads == heads
    assert np.array_equal(a.words, b.words)
    ref = orc.fasta_reads_ref(raw[:20000], 150)
    assert [h for h, _ in ref] == a.heads[:len(ref)]
    assert np.array_equal(np.stack([w for _, w in ref]), a.words[:len(ref)])


def _unpack(words: np.ndarray, nb: int) -> np.ndarray:
    return ((words[:, None] >> (2 * np.arange(16, dtype=np.uint32))) & 3).astype(np.uint8).reshape(-1)[:nb]


GENOME_CASES = [
    b"",
    b"no record\nACGT\n",
    b"junk\n>chr1 first\nACGTNacgtRYK\nTTTT\n>chr2\r\nGGGGCCCC\r\nAA\r\n>empty\n>last no newline\nACG",
    b">a\nACGT\r>b run-on header\nCCCC\n>c\nTT>G\n",      # '\r>' starts b inside a's sequence
    b">h1 header runs on\r>h2\nACGTACGT\n>h3\n" + b"A" * 33 + b"\n",  # h1's '\n' lies in h2
    b">only header",
]


@pytest.mark.parametrize("ci", range(len(GENOME_CASES)))
def test_genome_packer_matches_oracle(ci):
    raw = GENOME_CASES[ci]
    pack = rm.pack_reference(raw, nthreads=3)
    heads, seqs = orc.ref_table(raw)
    assert pack.heads == heads
    assert list(pack.nbases) == [len(q) for q in seqs]
    off = 0
    for r, q in enumerate(seqs):
        assert pack.word_off[r] == off
        nw = (len(q) + 15) // 16
        assert np.array_equal(pack.words[off:off + nw], orc.forward_pack(q, len(q)))
        assert pack.words[off + nw] == 0  # guard word
        off += nw + 1
    assert pack.words.size == max(off, 1)


def test_genome_packer_large_records_across_items_and_threads(tmp_path):
    """Records longer than the packer's 8 MB work items, odd line widths and
    CRLF: items split mid-record at every base alignment; the result does
    not depend on the thread count; a path source is read through mmap."""
    recs = synth.random_genome([21_000_000, 777, 9_000_001], seed=13, n_frac=0.02, run_min=10, run_max=5000)
    raw = synth.genome_fasta([">big one", ">small", ">mid"], recs, width=61)
    raw = raw.replace(b"\n", b"\r\n", 200_000)
    p = tmp_path / "g.fa"
    p.write_bytes(raw)
    a = rm.pack_reference(raw, nthreads=1)
    b = rm.pack_reference(str(p), nthreads=7)
    assert a.heads == b.heads == [">big one", ">small", ">mid"]
    assert np.array_equal(a.words, b.words) and np.array_equal(a.word_off, b.word_off)
    heads, seqs = orc.ref_table(raw)
    for r, q in enumerate(seqs):
        assert a.nbases[r] == len(q)
        assert np.array_equal(_unpack(a.words[a.word_off[r]:], len(q)), q)


def test_reference_windows_match_oracle():
    recs = synth.random_genome([700, 149, 150, 333, 2000], seed=4, n_frac=0.1, run_min=5, run_max=40)
    heads = [">A one", ">B", ">C", ">D", ">E"]
    fa = b"leading junk\n" + synth.genome_fasta(heads, recs, width=37).replace(b"T", b"t", 50)
    for k, kstep in ((150, 15), (150, 150), (50, 1), (17, 3)):
        pack = rm.pack_reference(fa)
        pos, rec, st = rm.window_positions(pack, k, kstep)
        ref = orc.ref_windows_ref(fa, k, kstep)
        assert len(ref) == pos.size
        W = (k + 15) // 16
        for i, (hd, start, words) in enumerate(ref):
            assert pack.heads[rec[i]] == hd and st[i] == start
            p = int(pos[i])
            q, sh = p >> 4, 2 * (p & 15)
            g = pack.words.astype(np.uint64)
            for j in range(W):
                v = (int(g[q + j]) >> sh) | ((int(g[q + j + 1]) << (32 - sh)) & 0xFFFFFFFF if sh else 0)
                v &= 0xFFFFFFFF
                if j == W - 1 and k & 15:
                    v &= (1 << (2 * (k & 15))) - 1
                assert v == int(words[j])


def test_batch_column_layout():
    col_win, strand = batch_column_order(10, 4)
    assert list(col_win) == [0, 1, 2, 3, 0, 1, 2, 3, 4, 5, 6, 7, 4, 5, 6, 7, 8, 9, 8, 9]
    assert list(strand) == [0] * 4 + [1] * 4 + [0] * 4 + [1] * 4 + [0, 0, 1, 1]


def test_index_container_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    N, rdim, m = 40, 64, 2  # rdim = 2*m*4^c with c = 2
    pack = rm.pack_records([">r1 a", ">r2"], [rng.integers(0, 4, 300, dtype=np.uint8),
                                             rng.integers(0, 4, 100, dtype=np.uint8)])
    idx = Index(format=rm.FP8_FORMAT, source="x.fa", k=20, kstep=2, s=5, m=m, c=2, normalize=0, n_frag=N // 2,
                embeds8=rng.integers(0, 256, (N, rdim), dtype=np.uint8),
                norms=rng.random((N, m), dtype=np.float32), rec_heads=pack.heads,
                col_rec=rng.integers(0, 2, N).astype(np.int32), starts=rng.integers(1, 99, N),
                strand=(np.arange(N) % 2).astype(np.uint8), col_pos=rng.integers(0, 999, N),
                genome=pack.words, rec_word_off=pack.word_off, rec_nbases=pack.nbases)
    p = tmp_path / "t.r2mi"
    idx.save(p)
    back = rm.load_index(str(p))
    for name in ("embeds8", "norms", "col_rec", "starts", "strand", "col_pos", "genome"):
        assert np.array_equal(np.asarray(getattr(back, name)), np.asarray(getattr(idx, name))), name
    assert back.rec_heads == idx.rec_heads and back.k == 20 and back.heads[0] == idx.heads[0]
    with pytest.raises(ValueError):
        bad = tmp_path / "bad.bin"
        bad.write_bytes(b"not an index at all")
        rm.load_index(str(bad))


@pytest.mark.parametrize("x,s", [(0.9873047, "0.9873047"), (1.0, "1.0"), (0.5, "0.5"), (-0.25, "-0.25"),
                                 (1e-5, "1.0e-5"), (0.0001, "0.0001"), (3.1415e-5, "3.1415e-5"),
                                 (123456.0, "123456.0"), (1e6, "1.0e6"), (0.1, "0.1"), (-1e-7, "-1.0e-7"),
                                 (0.0, "0.0"), (float("-inf"), "-Inf"), (0.0012345, "0.0012345"),
                                 (1.2345678e8, "1.2345678e8")])
def test_julia_float32_repr(x, s):
    assert rm.julia_repr_f32(x) == s


def test_parse_read_head_formats():
    h = rm.parse_read_head(">read_12 start=345 len=150 src=chrA extra words")
    assert h == dict(id=">read_12", start=345, len=150, src="chrA extra words")  # id keeps the ">"
    h = rm.parse_read_head(">NC_000001.11:80433546:false")
    assert h["start"] == 80433547 and h["len"] is None and h["src"] == "NC_000001.11"
    assert rm.parse_read_head(">NC_11:49059499:true#2")["start"] == 49059500
    for bad in ("read_1 start=1 len=2 src=a", ">read_1 start=x len=2 src=a", ">read_1 len=2 src=a",
                ">a:b:true", ">a:1:maybe", ">a:1", ">read_1 start=1 len=2"):
        assert rm.parse_read_head(bad) is None
    for h in (">read_3 start=10 len=150 src=chrB", ">chrQ:99:true"):
        assert rm.parse_read_head(h) == orc.parse_read_head(h)


def test_provenance_scoring_matches_oracle():
    rng = np.random.default_rng(5)
    k, N, ktop = 150, 600, 20
    rec_heads = [">chrA one", ">chrB"]
    col_rec = rng.integers(0, 2, N).astype(np.int32)
    starts = rng.integers(1, 5000, N)
    idx = Index(format=rm.FP8_FORMAT, source="", k=k, kstep=15, s=8, m=4, c=4, normalize=0, n_frag=N // 2,
                embeds8=np.zeros((N, 16), np.uint8), norms=np.zeros((N, 4), np.float32), rec_heads=rec_heads,
                col_rec=col_rec, starts=starts, strand=np.zeros(N, np.uint8), col_pos=np.zeros(N, np.int64),
                genome=np.zeros(1, np.uint32), rec_word_off=np.zeros(2, np.int64), rec_nbases=np.zeros(2, np.int64))
    heads, locs = [], []
    for i in range(300):
        src = "chrA" if i % 2 else "chrB"
        heads.append(f">read_{i} start={int(rng.integers(1, 5000))} len={k} src={src}")
        locs.append(rng.choice(N, ktop, replace=False) + 1)
    locs = np.array(locs)
    got = rm.score_provenance(heads, locs, idx, ktop)
    ref = orc.map_and_count_ref(heads, locs, idx.heads, list(starts), k, ktop)
    assert got[0] == ref[0] and got[1] == ref[1] and list(got[2]) == ref[2]
    assert got[3] == ref[3] and got[4] == ref[4]


def test_synth_even_sampler_and_packing():
    heads = [">g1 a", ">g2 b"]
    recs = synth.random_genome([5000, 3000], seed=1, gc=0.41, n_frac=0.05, run_min=20, run_max=100)
    reads, hd, rix, st = synth.sample_reads_even(heads, recs, 200, 150, 0.0, seed=3)
    assert len(reads) == 200 and list(synth.even_alloc([3, 1], 4)) == [3, 1]
    for r, h, j, s0 in zip(reads, hd, rix, st):
        codes, nmask = recs[j]
        assert not nmask[s0 - 1:s0 - 1 + 150].any()
        assert np.array_equal(r, codes[s0 - 1:s0 - 1 + 150])
        assert rm.parse_read_head(h)["start"] == s0
    w = synth.pack_reads(reads[:5], 150)
    for i in range(5):
        assert np.array_equal(w[i], orc.forward_pack(reads[i], 150))
    mutated = synth.substitute(np.zeros(100000, np.uint8), 0.05, np.random.default_rng(0))
    assert abs((mutated != 0).mean() - 0.05) < 0.005


def test_even_sampler_with_the_reference_draws():
    """model="reference": the reference sampler's draws (sample.jl:589-604):
    Xoshiro(seed), one child per read seeded by rand(rng, Int64), mutate on
    the child -- deterministic in the seed, length kept, err = 0 exact
    windows, and read i equal to mutate(window_i) on child i."""
    from rotormap import jlrandom
    heads = [">g1 a", ">g2 b"]
    recs = synth.random_genome([5000, 3000], seed=1)
    r0, hd0, rix, st = synth.sample_reads_even(heads, recs, 40, 150, 0.0, seed=5, model="reference")
    for r, j, s0 in zip(r0, rix, st):
        assert np.array_equal(r, recs[j][0][s0 - 1:s0 - 1 + 150])
    r5, hd5, _, _ = synth.sample_reads_even(heads, recs, 40, 150, 0.05, seed=5, model="reference")
    again, _, _, _ = synth.sample_reads_even(heads, recs, 40, 150, 0.05, seed=5, model="reference")
    other, _, _, _ = synth.sample_reads_even(heads, recs, 40, 150, 0.05, seed=6, model="reference")
    assert hd5 == hd0 and all(r.size == 150 for r in r5)
    assert all(np.array_equal(a, b) for a, b in zip(r5, again))
    assert not all(np.array_equal(a, b) for a, b in zip(r5, other))
    rng = jlrandom.Xoshiro(5)
    kids = [jlrandom.Xoshiro(rng.rand_i64()) for _ in range(40)]
    for i in (0, 17, 39):
        assert np.array_equal(r5[i], jlrandom.mutate(r0[i], 0.05, kids[i]))


def test_mutate_edits_follows_the_reference_model():
    """mutate (RotorMap/common/dna.jl:120-183): ceil(n*err) operations split
    floor(n_err/3) insertions, as many deletions, the rest substitutions; the
    length stays n; err = 0 is the identity; a substitution-only count (n_err
    < 3) changes exactly the drawn positions to other bases."""
    rng = np.random.default_rng(3)
    codes = rng.integers(0, 4, 5000).astype(np.uint8)
    assert np.array_equal(synth.mutate_edits(codes, 0.0, rng), codes)
    for err in (0.0001, 0.01, 0.1, 0.3, 0.5):
        out = synth.mutate_edits(codes, err, np.random.default_rng(7))
        assert out.size == codes.size and out.dtype == np.uint8 and out.max() <= 3
    out = synth.mutate_edits(codes, 2 / 5000, np.random.default_rng(9))  # n_err = 2: two substitutions
    diff = np.flatnonzero(out != codes)
    assert 1 <= diff.size <= 2
    a = synth.mutate_edits(codes, 0.2, np.random.default_rng(11))
    b = synth.mutate_edits(codes, 0.2, np.random.default_rng(11))
    assert np.array_equal(a, b)


def test_native_float_format_matches_oracle_on_random_bits():
    """r2m_format_f32 (the table's score field) against the oracle's
    restatement of Julia's string(::Float32) on random float32 bit patterns
    spanning every exponent, plus subnormals, extremes and the literals."""
    rng = np.random.default_rng(5)
    bits = rng.integers(0, 2 ** 32, 20_000, dtype=np.uint64).astype(np.uint32)
    xs = bits.view(np.float32)
    extra = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 1.1754944e-38, 3.4028235e38,
                      1e-4, 9.999999e-5, 1e6, 999999.94, 0.1, 0.3, 2.5, 100.0, 1e-5, 123456.0], np.float32)
    for x in np.concatenate([xs, extra]):
        assert rm.julia_repr_f32(x) == orc.julia_repr_f32_ref(x), (float(x), x.view(np.uint32))


@pytest.mark.parametrize("nb", [1, 37, 5000])
def test_native_table_matches_oracle(nb, tmp_path):
    """write_table (r2m_format_table, threaded above 2048 reads) writes the
    oracle's map.jl lines byte for byte, to text and to binary streams."""
    import io as _io
    from rotormap.mapping import write_table

    class Idx:
        pass
    rng = np.random.default_rng(nb)
    N, k = 50_000, 20
    idx = Idx()
    idx.strand = rng.integers(0, 2, N).astype(np.uint8)
    idx.starts = rng.integers(1, 10 ** 9, N).astype(np.int64)
    idx.col_rec = rng.integers(0, 3, N).astype(np.int32)
    idx.rec_heads = [">chr1 one", ">chrX", ">scaffold_7 len=5"]
    vals = (rng.standard_normal((nb, k)) * 10.0 ** rng.integers(-7, 8, (nb, k))).astype(np.float32)
    locs = rng.integers(1, N + 1, (nb, k)).astype(np.int32)
    heads = [f">read_{i} start={i} len=150 src=chr1" if i % 3 else f"noangle_{i}" for i in range(nb)]
    want = orc.table_lines_ref(vals, locs, heads, idx.strand, idx.starts, idx.col_rec, ["chr1", "chrX", "scaffold_7"])
    t = _io.StringIO()
    assert write_table(t, vals, locs, heads, idx) == nb * k
    assert t.getvalue() == want
    b = _io.BytesIO()
    write_table(b, vals, locs, heads, idx, nthreads=3)
    assert b.getvalue().decode() == want
    bad = locs.copy()
    bad[0, 0] = N + 1
    with pytest.raises(rm.R2MError):
        write_table(_io.BytesIO(), vals, bad, heads, idx)


def test_native_table_special_scores():
    """Scores the float formatter treats specially -- NaN, +-Inf, +-0,
    subnormals, the decimal/scientific boundaries -- in whole table lines,
    threaded, byte for byte as the oracle writes them."""
    import io as _io
    from rotormap.mapping import write_table

    class Idx:
        pass
    special = np.array([np.nan, np.inf, -np.inf, 0.0, -0.0, 1e-45, -1e-45, 1.1754942e-38, 1e-5, 9.999999e-5,
                        1e-4, 99999.99, 999999.94, 1e6, -1e6, 3.4028235e38, 0.1, -2.5], np.float32)
    rng = np.random.default_rng(17)
    nb, k, N = 3000, len(special), 1000
    idx = Idx()
    idx.strand = rng.integers(0, 2, N).astype(np.uint8)
    idx.starts = rng.integers(1, 10 ** 12, N).astype(np.int64)
    idx.col_rec = np.zeros(N, np.int32)
    idx.rec_heads = [">only"]
    vals = np.tile(special, (nb, 1))
    for r in range(nb):
        rng.shuffle(vals[r])
    locs = rng.integers(1, N + 1, (nb, k)).astype(np.int32)
    heads = [f">q{i}" for i in range(nb)]
    want = orc.table_lines_ref(vals, locs, heads, idx.strand, idx.starts, idx.col_rec, ["only"])
    b = _io.BytesIO()
    write_table(b, vals, locs, heads, idx, nthreads=4)
    assert b.getvalue().decode() == want


def test_native_table_buffers_reused_across_calls():
    """The writer's buffers are pooled between calls: tables of different
    sizes and thread counts, one after another (with a rejected call in
    between), are each exactly the oracle's lines -- nothing left over from
    an earlier, larger table."""
    import io as _io
    from rotormap.mapping import write_table

    class Idx:
        pass
    rng = np.random.default_rng(99)
    N, k = 20_000, 8
    idx = Idx()
    idx.strand = rng.integers(0, 2, N).astype(np.uint8)
    idx.starts = rng.integers(1, 10 ** 6, N).astype(np.int64)
    idx.col_rec = rng.integers(0, 2, N).astype(np.int32)
    idx.rec_heads = [">a", ">bb long name"]
    for nb, nt in ((6000, 8), (3, 1), (4100, 2), (6000, 8), (1, 4), (2500, 3)):
        vals = rng.uniform(-2, 2, (nb, k)).astype(np.float32)
        locs = rng.integers(1, N + 1, (nb, k)).astype(np.int32)
        heads = [f">r{nb}_{i}" + "x" * int(rng.integers(0, 40)) for i in range(nb)]
        want = orc.table_lines_ref(vals, locs, heads, idx.strand, idx.starts, idx.col_rec, ["a", "bb"])
        b = _io.BytesIO()
        write_table(b, vals, locs, heads, idx, nthreads=nt)
        assert b.getvalue().decode() == want
        if nb == 4100:
            bad = locs.copy()
            bad[-1, -1] = 0
            with pytest.raises(rm.R2MError):
                write_table(_io.BytesIO(), vals, bad, heads, idx, nthreads=nt)


def test_header_list_behaves_like_a_list():
    hs = [">a one", ">b", "", ">c three words", ">" + "x" * 300]
    blob = ("\n".join(hs) + "\n").encode()
    hl = rm.HeaderList.from_blob(blob)
    assert len(hl) == 5 and list(hl) == hs and hl == hs and hs == hl
    assert hl[0] == ">a one" and hl[-1] == hs[-1] and hl[2] == ""
    assert hl[1:4] == hs[1:4] and len(hl[1:4]) == 3 and hl[1:4].blob() == ("\n".join(hs[1:4]) + "\n").encode()
    assert hl[::2] == hs[::2] and hl[3:1] == [] and list(hl[5:]) == []
    with pytest.raises(IndexError):
        hl[5]
    f = rm.fasta_reads(b">r1 x\nACGT\n>r2\nAAAA\n", k=4)
    assert isinstance(f.heads, rm.HeaderList) and f.heads == [">r1 x", ">r2"]


@pytest.mark.parametrize("chunk", [1, 7, 64, 1000, 1 << 20])
def test_fasta_pieces_cut_at_record_starts(chunk):
    """The chunked readers' pieces: they concatenate to the input, every
    piece after the first starts a record, and parsing piece by piece gives
    the whole input's records (host reader; inputs without an unclosed
    header, where the two parses cannot differ)."""
    from rotormap.fasta import _fasta_pieces
    rng = np.random.default_rng(chunk)
    recs = []
    for r in range(60):
        n = int(rng.integers(0, 300))
        seq = synth.LETTERS[rng.integers(0, 4, n)].tobytes()
        eol = [b"\n", b"\r\n"][int(rng.integers(0, 2))]
        w = int(rng.integers(1, 90))
        recs.append(b">rec%d x>y\n" % r + eol.join(seq[i:i + w] for i in range(0, n, w)) + eol)
    raw = b"junk > line\n" + b"".join(recs)
    pieces = list(_fasta_pieces(raw, chunk))
    assert b"".join(pieces) == raw
    for p in pieces[1:]:
        assert p.startswith(b">")
    for k in (1, 100):
        whole = rm.fasta_reads(raw, k=k)
        parts = [rm.fasta_reads(p, k=k) for p in pieces]
        assert [h for f in parts for h in f.heads] == list(whole.heads)
        got = [f.words for f in parts if len(f)]
        assert np.array_equal(np.concatenate(got) if got else np.zeros((0, whole.words.shape[1]), np.uint32),
                              whole.words)


def test_package_modules_bind_every_name_they_load():
    """A static check of the host package (and bench.py): every name a
    module reads is bound somewhere in it (definition, import, assignment,
    argument) or is a builtin -- GPU-only code paths are covered too."""
    import ast
    import builtins
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    paths = sorted((root / "qpg-rotormap_b200" / "rotormap").glob("*.py")) + [root / "bench.py"]
    for path in paths:
        t = ast.parse(path.read_text())
        bound = set()
        for x in ast.walk(t):
            if isinstance(x, ast.Name) and isinstance(x.ctx, (ast.Store, ast.Del)):
                bound.add(x.id)
            elif isinstance(x, (ast.FunctionDef, ast.AsyncFunctionDef, ast.ClassDef)):
                bound.add(x.name)
            elif isinstance(x, ast.arg):
                bound.add(x.arg)
            elif isinstance(x, (ast.Import, ast.ImportFrom)):
                for a in x.names:
                    bound.add((a.asname or a.name).split(".")[0])
            elif isinstance(x, ast.ExceptHandler) and x.name:
                bound.add(x.name)
        used = {x.id for x in ast.walk(t) if isinstance(x, ast.Name) and isinstance(x.ctx, ast.Load)}
        missing = sorted(u for u in used if u not in bound and not hasattr(builtins, u)
                         and u not in ("__file__", "__name__"))
        assert not missing, f"{path.name}: {missing}"


def test_pick_reader_follows_the_faster_path(tmp_path, monkeypatch):
    """reader="auto": the host reader on a host with >= 8 threads for inputs
    up to 8 GiB, else the GPU reader (which streams any size)."""
    import os
    from rotormap.engine import pick_reader
    p = tmp_path / "r.fa"
    p.write_bytes(b">r\nACGT\n")
    assert pick_reader(str(p), "device") == "device" and pick_reader(str(p), "host") == "host"
    monkeypatch.setattr(os, "cpu_count", lambda: 16)
    assert pick_reader(str(p)) == "host" and pick_reader(b">r\nAC\n") == "host"
    assert pick_reader(str(tmp_path / "missing.fa")) == "device"
    monkeypatch.setattr(os, "cpu_count", lambda: 2)
    assert pick_reader(str(p)) == "device"
