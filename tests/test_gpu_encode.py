"""GPU parity of the encoder, reverse complement and e4m3 quantisers against
the CPU oracle (RotorMap/encode/kernel.jl:348-394 _check_frag_kernel_real,
index/build.jl:1040 _check_revcomp, search/engine_fp8.jl:603-617
_check_quantize_path are the reference's own versions of these checks)."""
import numpy as np
import pytest
import torch

from conftest import random_words
from oracle import oracle as orc

import rotormap as rm

pytestmark = pytest.mark.gpu

# FP32 embedding tolerance: |gpu - ref| <= RTOL*|ref| + ATOL (rows are unit
# energy, bins ~0.04; ATOL covers bins that cancel to ~0).
RTOL_F32 = 1e-5
ATOL_F32 = 2e-7
# against the fp64 golden encoder the fp32 phasors/sums add ~1e-7 per term
ATOL_F64 = 2e-6

CONFIGS = [
    (150, 8, 4, 4),   # the production read encoder (s8 m4 c4, 150 bp)
    (100, 8, 4, 4),   # batching-form index k
    (250, 8, 4, 4),
    (37, 5, 1, 3),
    (2001, 5, 1, 4),  # nw > 512: the reference thread recurrence
    (20, 8, 2, 2),
    (20000, 5, 1, 5),  # the reference's production encoder at the reader's default k
]


def _gpu_encode(words, re, normalize=0, dtype=torch.float32, scaled=False):
    dn = torch.from_numpy(words.reshape(-1).view(np.int32)).cuda()
    out = rm.encode_frag_real_batch_alloc(dtype, re, dn, normalize, scaled=scaled)
    torch.cuda.synchronize()
    return [t.cpu().numpy() if t is not None else None for t in out]


@pytest.mark.parametrize("k,s,m,c", CONFIGS)
@pytest.mark.parametrize("normalize", [0, 1, 2, 3])
def test_encoder_f32_vs_oracle(k, s, m, c, normalize):
    rng = np.random.default_rng(k * 31 + normalize)
    n = 64 if k < 1000 else 8
    words = random_words(rng, n, k)
    re = rm.RopeEncoder(k=k, s=s, m=m, c=c)
    emb, norms = _gpu_encode(words, re, normalize)
    o32, n32 = orc.rope_f32(words, k, s, m, c, normalize)
    o64, n64 = orc.rope_f64(words, k, s, m, c, normalize)
    heavy = normalize >= 2
    if heavy:
        # modes 2/3 map every nonzero bin z to z/(|z|+eps) (or /sqrt): a bin
        # whose phasors cancel to fp32 rounding residue (~1e-8) becomes a
        # unit-size value in one summation order and 0 in another.  Compare
        # the well-conditioned bins (raw |z| > 1e-3) only, as the reference
        # itself loosens these modes (kernel.jl:342-347).
        # The row norm of these modes counts every such bin, so rows holding
        # one are skipped whole.
        r0, rn0 = orc.rope_f64(words, k, s, m, c, 0)
        nb_ = r0.shape[1] // 2
        raw = np.hypot(r0[:, :nb_], r0[:, nb_:]) * rn0[:, :1]
        ok_rows = ~np.any((raw != 0) & (raw <= 1e-3), axis=1)
        assert ok_rows.mean() > 0.5
        emb, o32, o64 = emb[ok_rows], o32[ok_rows], o64[ok_rows]
        norms, n64 = norms[ok_rows], n64[ok_rows]
    rt, at = (RTOL_F32, ATOL_F32) if not heavy else (1e-4, 1e-5)
    np.testing.assert_allclose(emb, o32, rtol=rt, atol=at)
    np.testing.assert_allclose(emb, o64, rtol=rt, atol=ATOL_F64 if not heavy else 1e-4)
    rows = [0] if normalize == 0 else list(range(m))
    np.testing.assert_allclose(norms[:, rows], n64[:, rows], rtol=1e-5 if not heavy else 1e-4)
    if normalize == 0:
        e = (emb.astype(np.float64) ** 2).sum(axis=1)
        np.testing.assert_allclose(e, 1.0, rtol=1e-5)  # unit energy (stream.jl:276-288)
        # rows 2..m of norms hold the per-copy partial energies (kernel.jl:196)
        np.testing.assert_allclose(norms[:, 1:], n32[:, 1:], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("k,s,m,c", CONFIGS[:3])
def test_encoder_output_forms_are_the_quantised_f32(k, s, m, c):
    """fp16 / e4m3 / scaled-e4m3 outputs are exactly the oracle's conversions
    of the kernel's own fp32 values (bit-exact quantisation)."""
    rng = np.random.default_rng(5)
    words = random_words(rng, 200, k)
    re = rm.RopeEncoder(k=k, s=s, m=m, c=c)
    f32, _ = _gpu_encode(words, re)
    f16, _ = _gpu_encode(words, re, dtype=torch.float16)
    e8, _ = _gpu_encode(words, re, dtype=torch.uint8)
    s8, _, sc = _gpu_encode(words, re, dtype=torch.uint8, scaled=True)
    assert np.array_equal(f16.view(np.uint16), orc.f32_to_f16_bits(f32))
    assert np.array_equal(e8, orc.quantize_parity(f32))
    q, scale = orc.quantize_scaled(f32)
    assert np.array_equal(s8, q)
    assert np.array_equal(sc, scale)


def test_encoder_deterministic_and_batch_independent():
    rng = np.random.default_rng(9)
    re = rm.RopeEncoder(k=150, s=8, m=4, c=4)
    words = random_words(rng, 1000, 150)
    a, _ = _gpu_encode(words, re)
    b, _ = _gpu_encode(words, re)
    c, _ = _gpu_encode(words[:7], re)
    assert np.array_equal(a, b)
    assert np.array_equal(a[:7], c)


@pytest.mark.parametrize("k", list(range(1, 41)) + [150, 2001, 20000])
def test_revcomp_words_bit_exact(k):
    rng = np.random.default_rng(k)
    n = 16
    words = random_words(rng, n, k)
    d = torch.from_numpy(words.reshape(-1).view(np.int32)).cuda()
    out = torch.empty_like(d)
    rm.revcomp_frag_words(out, d, k, n)
    got = out.cpu().numpy().view(np.uint32).reshape(n, -1)
    for f in range(n):
        assert np.array_equal(got[f], orc.revcomp_words_ref(words[f], k))


def test_quantisers_exhaustive_fp16_and_random_fp32():
    h = np.arange(65536, dtype=np.uint32).astype(np.uint16).view(np.float16)
    finite = np.isfinite(h)
    src16 = torch.from_numpy(h[finite].copy()).cuda()
    dst = torch.empty(src16.numel(), dtype=torch.uint8, device="cuda")
    rm.f16_to_f8(dst, src16)
    ref = orc.f32_to_e4m3(h[finite].astype(np.float32))
    assert np.array_equal(dst.cpu().numpy(), ref)
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.standard_normal(1 << 20) * s for s in (1e-4, 1e-2, 1.0, 30.0, 1e3)]).astype(np.float32)
    x = np.concatenate([x, np.array([448.0, 464.0, 464.1, 480.0, -1e9, 2.0 ** -9, 2.0 ** -10,
                                     2.0 ** -10 * 1.0001, 0.0, -0.0], np.float32)])
    s32 = torch.from_numpy(x).cuda()
    d32 = torch.empty(x.size, dtype=torch.uint8, device="cuda")
    rm.f32_to_f8(d32, s32)
    assert np.array_equal(d32.cpu().numpy(), orc.f32_to_e4m3(x))


def test_ref_windows_columns_match_oracle():
    """GPU index columns (fwd + rc, batch layout) vs oracle windows."""
    from rotormap import synth
    recs = synth.random_genome([3000, 1234, 149, 700], seed=3, n_frac=0.05, run_min=10, run_max=60)
    heads = [">chrA one", ">chrB two", ">tiny", ">chrC"]
    fa = synth.genome_fasta(heads, recs, width=61).replace(b"ACG", b"acg", 3)
    k, kstep, batch = 150, 15, 64
    re = rm.RopeEncoder(k=k, s=8, m=4, c=4)
    pack = rm.pack_reference(fa)
    pos, rec, st = rm.window_positions(pack, k, kstep)
    wins = orc.ref_windows_ref(fa, k, kstep)
    assert len(wins) == pos.size
    assert [w[1] for w in wins] == list(st)
    nwin = pos.size
    g = torch.from_numpy(pack.words.view(np.int32)).cuda()
    p = torch.from_numpy(pos).cuda()
    out = torch.empty((2 * nwin, re.rdim), dtype=torch.float32, device="cuda")
    nrm = torch.empty((2 * nwin, re.m), dtype=torch.float32, device="cuda")
    from rotormap._lib import check, lib, ptr, OUT_F32
    check(lib().r2m_encode_ref_windows(ptr(out), OUT_F32, ptr(nrm), None, ptr(g), ptr(p), nwin, batch,
                                       k, 8, 4, 4, 0, torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    fw = np.stack([w[2] for w in wins])
    rcw = np.stack([orc.revcomp_words_ref(w, k) for w in fw])
    of, _ = orc.rope_f32(fw, k, 8, 4, 4)
    orr, _ = orc.rope_f32(rcw, k, 8, 4, 4)
    col_win, strand = rm.index.batch_column_order(nwin, batch)
    exp = np.where(strand[:, None] == 0, of[col_win], orr[col_win])
    np.testing.assert_allclose(got, exp, rtol=RTOL_F32, atol=ATOL_F32)
    # the e4m3 build is the parity quantisation of those fp32 columns
    idx = rm.build_index(re, fa, kstep=kstep, batch_size=batch)
    assert np.array_equal(idx.embeds8.cpu().numpy(), orc.quantize_parity(got))
    assert np.array_equal(idx.strand, strand)
    assert list(idx.starts) == list(st[col_win])


def test_reference_experiment_curves_through_the_gpu_encoder():
    """The reference's committed experiment outputs (k = 20,000, s5 m1 c5;
    tests/golden/rope_sweeps.json) reproduced by the GPU encoder's fp32 rows
    on the same Julia-seeded fixtures (rotormap.jlrandom): the shift
    sweep's anchor and 21 mutation-sweep points within 1e-5 of the
    reference's float64 inner products."""
    import json
    from pathlib import Path
    from rotormap import jlrandom, synth
    sw = json.loads((Path(__file__).parent / "golden" / "rope_sweeps.json").read_text())
    K, S, M, C = 20000, 5, 1, 5
    re = rm.RopeEncoder(k=K, s=S, m=M, c=C)
    frag = jlrandom.generate_reference(sw["fragment"]["n"], sw["fragment"]["seed"])
    shifted = jlrandom.mutate_shift(frag, 0.05, jlrandom.Xoshiro(42))
    rows = sw["sweeps"]["mutation"]["rows"][::50] + [sw["sweeps"]["mutation"]["rows"][-1]]
    muts = [frag, shifted] + [jlrandom.mutate(frag, err, jlrandom.Xoshiro(sw["copy_seed_base"] + i))
                              for i, err, _, _ in rows]
    words = synth.pack_reads(muts, K)
    g, _ = _gpu_encode(words, re)
    D = g.shape[1] // 2

    def ip(a, b):
        a = a.astype(np.float64)
        b = b.astype(np.float64)
        r = a @ b
        return r, np.hypot(r, a[:D] @ b[D:] - a[D:] @ b[:D])

    anchor = sw["sweeps"]["shift"]["rows"][0]
    assert np.allclose(ip(g[0], g[1]), anchor[2:], rtol=0, atol=1e-5)
    for j, (_, _, ip_re, ip_abs) in enumerate(rows):
        assert np.allclose(ip(g[0], g[j + 2]), (ip_re, ip_abs), rtol=0, atol=1e-5)


def test_reference_periodic_table_through_the_gpu_encoder():
    """The reference's periodic-fragment table (RotorMap/legacy/test/
    ropeperiod.jl, tests/golden/rope_sweeps.json: a 4,002-base Xoshiro(42)
    motif tiled to k = 20,000, whose copies nearly cancel) through the GPU
    encoder's fp32 rows on the Julia-exact fixtures: 11 of its rows within
    1e-5 (the table prints 6 decimals)."""
    import json
    from pathlib import Path
    from rotormap import jlrandom, synth
    per = json.loads((Path(__file__).parent / "golden" / "rope_sweeps.json").read_text())["periodic"]
    K = per["k"]
    re = rm.RopeEncoder(k=K, s=5, m=1, c=5)
    frag = jlrandom.periodic_fragment(K, per["period"], per["seed"])
    rows = [r for r in per["rows"] if r[0] % 5 == 0 and r[0] > 0] + [per["rows"][1]]
    muts = [frag] + [jlrandom.mutate(frag, err, jlrandom.Xoshiro(per["seed"] + i)) for i, err, _, _ in rows]
    g, _ = _gpu_encode(synth.pack_reads(muts, K), re)
    D = g.shape[1] // 2

    def ip(a, b):
        a = a.astype(np.float64)
        b = b.astype(np.float64)
        r = a @ b
        return r, np.hypot(r, a[:D] @ b[D:] - a[D:] @ b[:D])

    for j, (_, _, ip_re, ip_abs) in enumerate(rows):
        assert np.allclose(ip(g[0], g[j + 1]), (ip_re, ip_abs), rtol=0, atol=1e-5)


SPARSE_CONFIGS = [(150, 8, 4, 4), (100, 8, 4, 4), (250, 8, 4, 4), (37, 5, 1, 3), (20, 8, 2, 2), (60, 6, 8, 3)]


@pytest.mark.parametrize("k,s,m,c", SPARSE_CONFIGS)
def test_sparse_and_dense_encoders_agree(k, s, m, c, monkeypatch):
    """The slot-based encoder (normalize 0, the default at read length) and
    the dense-histogram encoder form every bin as the same sum in the same
    order: fp32 rows agree to the rounding of the norm's summation order,
    and each path's fp16 / e4m3 outputs are the conversions of its own fp32
    values."""
    rng = np.random.default_rng(k + 7 * m)
    words = random_words(rng, 300, k)
    re = rm.RopeEncoder(k=k, s=s, m=m, c=c)
    outs = {}
    for path in ("sparse", "dense"):
        monkeypatch.setenv("R2M_ENCODER", path)
        f32, n32 = _gpu_encode(words, re)
        e8, _ = _gpu_encode(words, re, dtype=torch.uint8)
        s8, _, sc = _gpu_encode(words, re, dtype=torch.uint8, scaled=True)
        q, scale = orc.quantize_scaled(f32)
        if path == "dense" or 4 * m <= 16:
            assert np.array_equal(e8, orc.quantize_parity(f32))
            assert np.array_equal(s8, q) and np.array_equal(sc, scale)
        else:
            # fp32 rows wider than 16 bytes per c-mer run (m = 8) take the
            # dense path, whose norm sums in another order: the sparse path's
            # scales match to rounding, its bytes wherever that rounding does
            # not cross an e4m3 rounding boundary
            np.testing.assert_allclose(sc, scale, rtol=2e-6)
            assert np.mean(s8 != q) < 1e-4 and np.mean(e8 != orc.quantize_parity(f32)) < 1e-4
        outs[path] = (f32, n32)
    (a, na), (b, nb) = outs["sparse"], outs["dense"]
    np.testing.assert_allclose(a, b, rtol=2e-6, atol=1e-8)
    np.testing.assert_allclose(na, nb, rtol=2e-6)
    o32, _ = orc.rope_f32(words, k, s, m, c)
    np.testing.assert_allclose(a, o32, rtol=RTOL_F32, atol=ATOL_F32)


def test_sparse_index_windows_equal_dense(monkeypatch):
    """Index columns (forward and reverse complement from the packed
    genome, register-formed on the sparse path) from both encoders."""
    from rotormap import synth
    from rotormap._lib import OUT_E4M3_SCALED, check, lib, ptr
    recs = synth.random_genome([5000, 777, 3000], seed=4, n_frac=0.02, run_min=10, run_max=40)
    heads = [">a", ">b", ">c"]
    fa = synth.genome_fasta(heads, recs)
    for k in (150, 100, 37):
        pack = rm.pack_reference(fa)
        pos, _, _ = rm.window_positions(pack, k, 7)
        nwin = pos.size
        g = torch.from_numpy(pack.words.view(np.int32)).cuda()
        p = torch.from_numpy(pos).cuda()
        res = {}
        for path in ("sparse", "dense"):
            monkeypatch.setenv("R2M_ENCODER", path)
            out = torch.empty((2 * nwin, 2048), dtype=torch.uint8, device="cuda")
            nrm = torch.empty((2 * nwin, 4), dtype=torch.float32, device="cuda")
            sc = torch.empty((2 * nwin,), dtype=torch.float32, device="cuda")
            check(lib().r2m_encode_ref_windows(ptr(out), OUT_E4M3_SCALED, ptr(nrm), ptr(sc), ptr(g), ptr(p), nwin,
                                               100, k, 8, 4, 4, 0, torch.cuda.current_stream().cuda_stream))
            torch.cuda.synchronize()
            res[path] = (out.cpu().numpy(), nrm.cpu().numpy(), sc.cpu().numpy())
        (a, na, sa), (b, nb, sb) = res["sparse"], res["dense"]
        np.testing.assert_allclose(na, nb, rtol=2e-6)
        np.testing.assert_allclose(sa, sb, rtol=2e-6)
        # a norm rounded differently can move a value across an e4m3 rounding
        # boundary: at most one step, in a tiny share of the bytes
        diff = a != b
        assert diff.mean() < 1e-4
        t = orc.e4m3_table()
        assert np.all(np.abs(t[a[diff]] - t[b[diff]]) <= np.abs(t[b[diff]]) * 0.13 + 1e-9)
