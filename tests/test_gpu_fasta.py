"""Device FASTA reader (r2m_fasta_reads_device) against the oracle's restatement
of RotorMap/fasta/reader.jl and the host reader: identical records, words and
headers, bit for bit."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc

import rotormap as rm
from rotormap import synth

from test_cpu_host import FASTA_CASES

pytestmark = pytest.mark.gpu


def _check(raw: bytes, k: int, src=None):
    got = rm.fasta_reads_device(raw if src is None else src, k=k)
    ref = orc.fasta_reads_ref(raw, k) if len(raw) < 200_000 else None
    host = rm.fasta_reads(raw, k=k)
    w = got.words.cpu().numpy().view(np.uint32)
    assert got.heads == host.heads
    assert np.array_equal(w, host.words)
    if ref is not None:
        assert got.heads == [h for h, _ in ref]
        if ref:
            assert np.array_equal(w, np.stack([x for _, x in ref]))
    return got


@pytest.mark.parametrize("k", [1, 5, 16, 17, 31, 32, 33, 150])
@pytest.mark.parametrize("ci", range(len(FASTA_CASES)))
def test_device_reader_matches_oracle(ci, k):
    _check(FASTA_CASES[ci], k)


@pytest.mark.parametrize("seed", range(6))
def test_device_reader_random_layouts(seed):
    rng = np.random.default_rng(seed)
    alphabet = np.frombuffer(b"ACGTacgtNRYn-*", np.uint8)
    out = [b"preamble\n"] if seed % 2 else []
    for r in range(300):
        n = int(rng.integers(0, 400))
        seq = alphabet[rng.integers(0, alphabet.size, n)]
        eol = [b"\n", b"\r\n", b"\r"][int(rng.integers(0, 3))] if seed >= 3 else b"\n"
        width = int(rng.integers(1, 140))
        body = eol.join(seq[i:i + width].tobytes() for i in range(0, n, width))
        hdr_eol = b"\r\n" if eol == b"\r\n" else b"\n"
        out.append(b">rec%d %d" % (r, n) + hdr_eol + body + eol)
    raw = b"".join(out)
    for k in (1, 16, 17, 150, 333):
        _check(raw, k)


def test_device_reader_long_records_flush_the_staging_buffer():
    """k far above the 1 KB per-warp staging buffer, wrapped lines."""
    recs = synth.random_genome([30_000, 5_000, 20_000, 20_001, 19_999], seed=3, n_frac=0.05, run_min=10,
                               run_max=200)
    heads = [">long%d" % i for i in range(len(recs))]
    for width in (60, 1000, 100_000):
        raw = synth.genome_fasta(heads, recs, width=width)
        for k in (1000, 1023, 1025, 20_000):
            _check(raw, k)


def test_device_reader_many_tiles_and_unclosed_header():
    """Record starts spread over thousands of 4 KB tiles; an unclosed header
    far into the input drops it and every later record."""
    rng = np.random.default_rng(11)
    codes = rng.integers(0, 4, (60_000, 150), dtype=np.uint8)
    recs = [b">r%d len=150\n" % i + synth.LETTERS[c].tobytes() + b"\n" for i, c in enumerate(codes)]
    raw = b"".join(recs)
    g = _check(raw, 150)
    assert len(g) == 60_000
    # a '>' straight after the header text is part of the header ...
    run_on = b"".join(recs[:41_234]) + b">open header" + b"".join(recs[41_234:])
    g = _check(run_on, 150)
    assert len(g) == 60_000 and g.heads[41_234] == ">open header>r41234 len=150"
    # ... after a lone '\r' it starts the next record, leaving the header unclosed
    cut = b"".join(recs[:41_234]) + b">open header\r" + b"".join(recs[41_234:])
    g = _check(cut, 150)
    assert len(g) == 41_234


def test_device_reader_multi_block_scans():
    """More than 64K records: the kept-flag and header-length scans take the
    three-pass multi-block form; short records are skipped along the way."""
    rng = np.random.default_rng(12)
    n = 150_000
    lens = rng.integers(30, 50, n)
    codes = rng.integers(0, 4, int(lens.sum()), dtype=np.uint8)
    offs = np.r_[0, np.cumsum(lens)]
    raw = b"".join(b">q%d\n" % i + synth.LETTERS[codes[offs[i]:offs[i + 1]]].tobytes() + b"\n" for i in range(n))
    g = _check(raw, 40)
    assert len(g) == int((lens >= 40).sum()) and len(g) > 65_536


def test_device_reader_device_sources_any_alignment():
    recs = synth.random_genome([300] * 500, seed=8)
    raw = synth.genome_fasta([">s%d" % i for i in range(500)], recs, width=77)
    for shift in (0, 1, 3, 8, 15):
        buf = torch.zeros(len(raw) + 32, dtype=torch.uint8, device="cuda")
        buf[shift:shift + len(raw)] = torch.frombuffer(bytearray(raw), dtype=torch.uint8).cuda()
        _check(raw, 200, src=buf[shift:shift + len(raw)])


def test_device_reader_feeds_the_encoder():
    """Words parsed on the device encode exactly like host-parsed words."""
    recs = synth.random_genome([10_000], seed=2)
    reads, heads, _, _ = synth.sample_reads_even([">g"], recs, 300, 150, 0.02, seed=4)
    raw = synth.reads_fasta(heads, reads)
    re = rm.RopeEncoder(k=150, s=8, m=4, c=4)
    g = rm.fasta_reads_device(raw, k=150)
    h = rm.fasta_reads(raw, k=150)
    a = rm.encode_frag_real_batch_alloc(torch.float32, re, g.words)
    b = rm.encode_frag_real_batch_alloc(torch.float32, re, torch.from_numpy(h.words.view(np.int32)).cuda())
    assert torch.equal(a[0], b[0])


def test_device_reader_rejects_bad_arguments():
    with pytest.raises(ValueError):
        rm.fasta_reads_device(b">a\nACGT\n", k=0)
    with pytest.raises(ValueError):
        rm.fasta_reads_device(torch.zeros(4, dtype=torch.int32, device="cuda"), k=4)
    assert len(rm.fasta_reads_device(b"", k=4)) == 0


@pytest.mark.parametrize("chunk", [50, 999, 10_000, 1 << 30])
def test_device_reader_in_pieces_equals_whole_input(chunk):
    """fasta_chunks_device (the file in pieces cut at record starts) yields
    the whole-input records, and stops at an unclosed header exactly where
    the whole-input reader does."""
    rng = np.random.default_rng(chunk % 1000)
    recs = []
    for r in range(400):
        n = int(rng.integers(100, 200))
        seq = synth.LETTERS[rng.integers(0, 4, n)].tobytes()
        eol = [b"\n", b"\r\n"][int(rng.integers(0, 2))]
        recs.append(b">r%d\n" % r + seq[:70] + eol + seq[70:] + eol)
    for raw in (b"".join(recs), b"".join(recs[:250]) + b">open\r" + b"".join(recs[250:])):
        whole = rm.fasta_reads_device(raw, k=120)
        pieces = list(rm.fasta_chunks_device(raw, k=120, chunk_bytes=chunk))
        assert [h for p in pieces for h in p.heads] == list(whole.heads)
        assert torch.equal(torch.cat([p.words for p in pieces]), whole.words)
        assert pieces[-1].stopped == whole.stopped


def test_stream_in_small_pieces_equals_host_reader(tmp_path):
    """rope_topk_stream over a file read in small pieces: the same batches
    (numbering included) as the whole-input host reader."""
    heads = [">g1"]
    recs = synth.random_genome([40_000], seed=3)
    re = rm.RopeEncoder(k=150, s=8, m=4, c=4)
    idx = rm.build_index(re, synth.genome_fasta(heads, recs), kstep=15)
    reads, hd, _, _ = synth.sample_reads_even(heads, recs, 500, 150, 0.05, seed=9)
    p = tmp_path / "r.fa"
    p.write_bytes(synth.reads_fasta(hd, reads))
    a = list(rm.rope_topk_stream(re, str(p), idx.embeds8, k=20, batch_size=128, reader="device", chunk_bytes=7000))
    b = list(rm.rope_topk_stream(re, str(p), idx.embeds8, k=20, batch_size=128, reader="host"))
    assert [h for x in a for h in x.heads] == [h for x in b for h in x.heads] == hd
    va = np.concatenate([x.vals for x in a]); vb = np.concatenate([x.vals for x in b])
    la = np.concatenate([x.locs for x in a]); lb = np.concatenate([x.locs for x in b])
    assert np.array_equal(va, vb) and np.array_equal(la, lb)
    firsts = [x.first for x in a]
    assert firsts[0] == 1 and all(f2 - f1 == len(x.heads) for f1, f2, x in zip(firsts, firsts[1:], a))
