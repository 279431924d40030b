"""The reference's index .bin (Julia Serialization of the NamedTuple of
RotorMap/index/build.jl:755-772): reader and writer against the
hand-assembled fixture, round trips, and load_index's checks
(RotorMap/index/load.jl:49-73)."""
import struct
import sys
from pathlib import Path

import numpy as np
import pytest

import rotormap as rm
from rotormap import jlbin
from rotormap._lib import R2MError

GOLD = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLD))
import make_jlbin_fixture as FX  # noqa: E402


def _fixture_fields():
    emb = np.frombuffer(FX.EMBEDS8, np.uint8).reshape(FX.N, FX.RDIM)
    return [("format", FX.FORMAT), ("source", FX.SOURCE), ("k", FX.K), ("kstep", FX.KSTEP), ("s", FX.S),
            ("m", FX.M), ("c", FX.C), ("normalize", 0), ("fp8", True), ("n_frag", FX.N // 2),
            ("embeds8", jlbin.E4M3(emb)), ("norms", np.array(FX.NORMS, np.float32).reshape(FX.N, FX.M)),
            ("heads", FX.HEADS), ("starts", np.array(FX.STARTS, np.int64)),
            ("strand", np.array(FX.STRAND, np.uint8))]


def test_fixture_bytes_are_current():
    assert (GOLD / "index_tiny.bin").read_bytes() == FX.build()


def test_reader_decodes_the_hand_assembled_fixture():
    d, ver = jlbin.read_bin(GOLD / "index_tiny.bin")
    assert ver == 20
    assert list(d) == ["format", "source", "k", "kstep", "s", "m", "c", "normalize", "fp8", "n_frag",
                       "embeds8", "norms", "heads", "starts", "strand"]
    assert d["format"] == FX.FORMAT and d["source"] == FX.SOURCE
    assert (d["k"], d["kstep"], d["s"], d["m"], d["c"], d["normalize"], d["n_frag"]) == (20, 2, 3, 1, 1, 0, 2)
    assert d["fp8"] is True
    assert isinstance(d["embeds8"], jlbin.E4M3Array) and d["embeds8"].shape == (4, 8)
    assert bytes(np.asarray(d["embeds8"]).tobytes()) == FX.EMBEDS8
    assert d["norms"].dtype == np.float32 and d["norms"].ravel().tolist() == FX.NORMS
    assert d["heads"].tolist() == FX.HEADS and d["heads"].uniq == [">chrA tiny", ">B"]
    assert d["starts"].tolist() == FX.STARTS and d["strand"].tolist() == FX.STRAND


def test_writer_reproduces_the_fixture_bytes(tmp_path):
    p = tmp_path / "w.bin"
    jlbin.write_bin(p, _fixture_fields())
    assert p.read_bytes() == (GOLD / "index_tiny.bin").read_bytes()


def test_load_index_of_the_fixture():
    idx = rm.load_index(GOLD / "index_tiny.bin")
    assert idx.format == rm.FP8_FORMAT and idx.N == 4 and idx.rdim == 8
    assert idx.heads == FX.HEADS and idx.rec_heads == [">chrA tiny", ">B"]
    assert np.asarray(idx.starts).tolist() == FX.STARTS and np.asarray(idx.strand).tolist() == FX.STRAND
    assert np.asarray(idx.embeds8).tobytes() == FX.EMBEDS8
    assert idx.genome is None  # the reference's file carries no packed genome


def _random_index(rng, N=64, m=2, c=2, nrec=3, scaled=False):
    rdim = 2 * m * 4 ** c
    heads = [f">rec{i} some description {i}" for i in range(nrec)] + [">s"]
    col_rec = rng.integers(0, len(heads), N).astype(np.int32)
    return rm.Index(format=rm.SCALED_FORMAT if scaled else rm.FP8_FORMAT, source="/x/genome.fa", k=30, kstep=3,
                    s=5, m=m, c=c, normalize=0, n_frag=N // 2,
                    embeds8=rng.integers(0, 256, (N, rdim), dtype=np.uint8),
                    norms=rng.random((N, m), dtype=np.float32), rec_heads=heads, col_rec=col_rec,
                    starts=rng.integers(1, 10 ** 6, N), strand=(np.arange(N) % 2).astype(np.uint8),
                    col_pos=np.zeros(N, np.int64), genome=np.zeros(1, np.uint32),
                    rec_word_off=np.zeros(len(heads), np.int64), rec_nbases=np.zeros(len(heads), np.int64),
                    scales=rng.random(N, dtype=np.float32) if scaled else None)


@pytest.mark.parametrize("scaled", [False, True])
def test_save_load_round_trip(tmp_path, scaled):
    rng = np.random.default_rng(3)
    idx = _random_index(rng, scaled=scaled)
    p = tmp_path / "i.bin"
    idx.save(p)
    assert jlbin.is_julia_stream(p)
    back = rm.load_index(p)
    assert back.format == idx.format and (back.k, back.kstep, back.s, back.m, back.c) == (30, 3, 5, 2, 2)
    for name in ("embeds8", "norms", "starts", "strand"):
        assert np.array_equal(np.asarray(getattr(back, name)), np.asarray(getattr(idx, name))), name
    assert back.heads == idx.heads
    if scaled:
        assert np.array_equal(np.asarray(back.scales), idx.scales)
    # repeated headers are written once: the file is far smaller than the
    # headers written out in full for every column
    full = sum(len(h) for h in idx.heads)
    assert p.stat().st_size < idx.embeds8.nbytes + idx.norms.nbytes + 9 * idx.N * 2 + full


def test_wide_back_reference_ids(tmp_path):
    """More than 65,535 shared strings: later references need the 4-byte
    BACKREF form."""
    n = 70_000
    uniq = [f">record_{i:06d}" for i in range(n)]
    idx = np.concatenate([np.arange(n), np.arange(n)[::-1]]).astype(np.int32)
    p = tmp_path / "wide.bin"
    jlbin.write_bin(p, [("heads", jlbin.StrVec(uniq, idx)), ("n", n)])
    raw = p.read_bytes()
    assert bytes([42]) + struct.pack("<i", 70_000) in raw  # BACKREF tag + Int32 id
    d, _ = jlbin.read_bin(p)
    assert d["n"] == n and d["heads"].uniq == uniq and np.array_equal(d["heads"].idx, idx)


def test_long_strings_symbols_and_integers(tmp_path):
    src = "/" + "d" * 300 + "/ref.fa"  # > 255 bytes: LONGSTRING
    vals = [-5, 0, 32, 33, 2 ** 31 - 1, 2 ** 31, -(2 ** 31), -(2 ** 31) - 1, 2 ** 62]
    fields = [("source", src), ("a_field_name_longer_than_7", True), ("flag", False)]
    fields += [(f"i{j}", v) for j, v in enumerate(vals)]
    p = tmp_path / "s.bin"
    jlbin.write_bin(p, fields)
    d, _ = jlbin.read_bin(p)
    assert d["source"] == src and d["a_field_name_longer_than_7"] is True and d["flag"] is False
    assert [d[f"i{j}"] for j in range(len(vals))] == vals


def test_julia_int64_encodings(tmp_path):
    p = tmp_path / "e.bin"
    jlbin.write_bin(p, [("a", 7), ("b", 1000), ("c", 2 ** 40)])
    raw = p.read_bytes()
    assert bytes([223 + 7]) in raw                                # literal
    assert bytes([49]) + struct.pack("<i", 1000) in raw           # SHORTINT64
    assert bytes([8]) + struct.pack("<q", 2 ** 40) in raw         # INT64


def test_row_layout_index_loads(tmp_path):
    """The classic row layout (format "indexreal.v1", fp16 rows (N, rdim))."""
    rng = np.random.default_rng(4)
    N, m, c = 6, 1, 1
    rdim = 2 * m * 4 ** c
    rows = rng.standard_normal((rdim, N)).astype(np.float16)  # Julia (N, rdim), column-major
    p = tmp_path / "rows.bin"
    jlbin.write_bin(p, [("format", "indexreal.v1"), ("source", "x.fa"), ("k", 20), ("kstep", 2), ("s", 3),
                        ("m", m), ("c", c), ("normalize", 0), ("fp16", True), ("n_frag", N // 2),
                        ("embeds", rows), ("norms", np.ones((N, m), np.float32)),
                        ("heads", [">a"] * N), ("starts", np.arange(1, N + 1)),
                        ("strand", np.zeros(N, np.uint8))])
    idx = rm.load_index(p)
    assert idx.embeds8 is None and idx.rows.shape == (rdim, N) and np.array_equal(idx.rows, rows)


def test_legacy_format_tag_loads(tmp_path):
    fields = _fixture_fields()
    fields[0] = ("format", "indexflowreal.fp8.v1")
    p = tmp_path / "legacy.bin"
    jlbin.write_bin(p, fields)
    assert rm.load_index(p).N == 4


@pytest.mark.parametrize("change,msg", [
    (("format", "something.v9"), "not an indexreal"),
    (("normalize", 1), "normalize = 0"),
    (("n_frag", 3), "shape mismatch"),
    (("starts", np.arange(3, dtype=np.int64)), "meta length mismatch"),
    (("embeds8", np.zeros((4, 8), np.uint8)), "eltype mismatch"),
])
def test_load_index_checks(tmp_path, change, msg):
    fields = [change if n == change[0] else (n, v) for n, v in _fixture_fields()]
    p = tmp_path / "bad.bin"
    jlbin.write_bin(p, fields)
    with pytest.raises(ValueError, match=msg):
        rm.load_index(p)


def test_truncated_and_foreign_streams(tmp_path):
    raw = (GOLD / "index_tiny.bin").read_bytes()
    for cut in (1, 9, 60, len(raw) - 1):
        p = tmp_path / f"cut{cut}.bin"
        p.write_bytes(raw[:cut])
        with pytest.raises(R2MError, match="index .bin"):
            jlbin.read_bin(p)
    p = tmp_path / "foreign.bin"
    p.write_bytes(bytes([55]) + b"JL" + bytes([20, 4, 0, 0, 0]) + bytes([22, 1, 2]))  # an Expr
    with pytest.raises(R2MError, match="unsupported tag 22"):
        jlbin.read_bin(p)
    p = tmp_path / "notjulia.bin"
    p.write_bytes(b"hello world")
    with pytest.raises(ValueError, match="not an"):
        rm.load_index(p)
    with pytest.raises(FileNotFoundError):
        rm.load_index(tmp_path / "missing.bin")


def test_container_still_written_for_r2mi(tmp_path):
    rng = np.random.default_rng(5)
    idx = _random_index(rng)
    p = tmp_path / "c.r2mi"
    idx.save(p)
    assert not jlbin.is_julia_stream(p)
    back = rm.load_index(p)
    assert np.array_equal(np.asarray(back.embeds8), idx.embeds8) and back.genome is not None


def test_attach_genome_from_source(tmp_path):
    """A .bin carries no packed genome; rescoring gets it from the source
    FASTA: each column's window position is found again."""
    from rotormap import synth
    heads = [">chrA one", ">chrB two"]
    recs = synth.random_genome([400, 300], seed=9)
    fa = tmp_path / "g.fa"
    fa.write_bytes(synth.genome_fasta(heads, recs))
    pack = rm.pack_reference(str(fa))
    pos, rec, st = rm.window_positions(pack, 50, 7)
    idx = _random_index(np.random.default_rng(1), N=2 * pos.size, nrec=2)
    idx.rec_heads, idx.source = heads, str(fa)
    idx.col_rec = np.concatenate([rec, rec]).astype(np.int32)
    idx.starts = np.concatenate([st, st])
    idx.k, idx.genome, idx.col_pos = 50, None, None
    rm.attach_genome(idx)
    assert np.array_equal(idx.col_pos, np.concatenate([pos, pos])) and np.array_equal(idx.genome, pack.words)


@pytest.mark.parametrize("body", [
    bytes([45]) + struct.pack("<i", 2_000_000_000),                        # LONGTUPLE of 2e9 items
    bytes([21, 0, 8, 20, 2, 49]) + struct.pack("<i", 2**30) + bytes([49]) + struct.pack("<i", 2**30),  # Int64 2^30 x 2^30
    bytes([21, 0, 33, 8]) + struct.pack("<q", 2**62),                       # String vector of 2^62
    bytes([21, 0, 13, 8]) + struct.pack("<q", 2**61),                       # Float32 vector: size overflows
    bytes([48]) + struct.pack("<i", -5),                                    # negative string length
])
def test_hostile_sizes_are_refused_not_trusted(tmp_path, body):
    """Counts and dims far beyond the stream's length fail with a parse
    error before any allocation or read trusts them."""
    p = tmp_path / "h.bin"
    p.write_bytes(bytes([55]) + b"JL" + bytes([20, 4, 0, 0, 0]) + body)
    with pytest.raises(R2MError, match="index .bin"):
        jlbin.read_bin(p)
