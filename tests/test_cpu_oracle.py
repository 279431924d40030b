"""CPU checks of the oracle itself: golden vectors, published encodings and
the reference's own known-answer properties.  No GPU is needed."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from conftest import random_words
from oracle import oracle as orc

GOLDEN = json.loads((Path(__file__).parent / "golden" / "rope_golden.json").read_text())
CODE = {"A": 0, "C": 1, "G": 2, "T": 3}


def golden_words(case):
    codes = np.array([CODE[case["unit"][j % len(case["unit"])]] for j in range(case["k"])], np.uint8)
    return orc.forward_pack(codes, case["k"])[None, :]


def golden_dense(case):
    nbin = case["nbin"]
    out = np.zeros(2 * nbin)
    for b, (re, im) in case["bins"].items():
        out[int(b)] = re
        out[nbin + int(b)] = im
    return out


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_oracle_f64_matches_closed_form(case):
    w = golden_words(case)
    out, norms = orc.rope_f64(w, case["k"], case["s"], case["m"], case["c"], 0)
    np.testing.assert_allclose(out[0], golden_dense(case), rtol=0, atol=1e-12)
    assert math.isclose(norms[0, 0], case["norm"], rel_tol=1e-12)


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_oracle_f32_matches_closed_form(case):
    w = golden_words(case)
    out, norms = orc.rope_f32(w, case["k"], case["s"], case["m"], case["c"], 0)
    # periodic fragments pour ~nw/P windows into each bin: fp32 summation
    # error grows with the window count
    nw = case["k"] - case["s"] + 1
    np.testing.assert_allclose(out[0], golden_dense(case), rtol=1e-5, atol=2e-6 * max(1.0, nw / 150))


# OCP FP8 E4M3 (bias 7, max 448, NaN = S.1111.111, no Inf): value -> byte
E4M3_KNOWN = [
    (0.0, 0x00), (-0.0, 0x80), (1.0, 0x38), (-1.0, 0xB8), (1.5, 0x3C), (2.0, 0x40), (3.0, 0x44),
    (448.0, 0x7E), (-448.0, 0xFE), (240.0, 0x77), (256.0, 0x78), (2.0 ** -6, 0x08),
    (2.0 ** -9, 0x01), (7 * 2.0 ** -9, 0x07), (0.875, 0x36),
    (1.0625, 0x38),     # tie between 1.0 and 1.125 -> even mantissa (1.0)
    (1.1875, 0x3A),     # tie between 1.125 and 1.25 -> even (1.25)
    (500.0, 0x7E), (1e9, 0x7E), (float("inf"), 0x7E), (-1e9, 0xFE),  # satfinite
    (2.0 ** -11, 0x00), (2.0 ** -10, 0x00),  # below / at half the smallest subnormal
    (3 * 2.0 ** -11, 0x01), (2.0 ** -10 * 1.0001, 0x01),
    (464.0, 0x7E),      # tie 448/480 -> 480 overflows -> saturates
]


@pytest.mark.parametrize("x,b", E4M3_KNOWN)
def test_e4m3_known_encodings(x, b):
    assert orc.f32_to_e4m3(np.array([x], np.float32))[0] == b


def test_e4m3_decode_table_and_round_trip():
    t = orc.e4m3_table()
    for b in range(256):
        s, e, m = b >> 7, (b >> 3) & 15, b & 7
        if e == 15 and m == 7:
            assert math.isnan(t[b])
            continue
        v = (m / 8.0) * 2.0 ** -6 if e == 0 else (1 + m / 8.0) * 2.0 ** (e - 7)
        assert t[b] == (-v if s else v)
        assert orc.f32_to_e4m3(np.array([t[b]], np.float32))[0] == b


def test_fp16_rounding_matches_ieee():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(1 << 18) * s for s in (1e-7, 1e-5, 1e-3, 1, 1e3, 6e4)])
    x = np.concatenate([x, [65504.0, 65519.0, 65520.0, 2.0 ** -24, 2.0 ** -25, 3 * 2.0 ** -26,
                            2.0 ** -14, 2.0 ** -14 - 2.0 ** -25]]).astype(np.float32)
    got = orc.f32_to_f16_bits(x)
    ref = x.astype(np.float16).view(np.uint16)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("k,s,m,c", [(150, 8, 4, 4), (37, 5, 1, 3), (2001, 5, 1, 4), (20, 8, 2, 2)])
def test_oracle_f32_tracks_f64_and_unit_energy(k, s, m, c):
    rng = np.random.default_rng(k)
    w = random_words(rng, 32, k)
    o64, n64 = orc.rope_f64(w, k, s, m, c, 0)
    o32, n32 = orc.rope_f32(w, k, s, m, c, 0)
    np.testing.assert_allclose(o32, o64, rtol=1e-5, atol=2e-6)
    np.testing.assert_allclose((o64 ** 2).sum(axis=1), 1.0, rtol=1e-12)
    np.testing.assert_allclose(n32[:, 0], n64[:, 0], rtol=1e-5)


def test_revcomp_reference_identities():
    rng = np.random.default_rng(1)
    for k in (1, 7, 16, 17, 150):
        w = random_words(rng, 4, k)
        for f in range(4):
            rc = orc.revcomp_words_ref(w[f], k)
            assert np.array_equal(orc.revcomp_words_ref(rc, k), w[f])
            codes = orc.frag_codes(w[f], k)
            assert np.array_equal(orc.frag_codes(rc, k), (3 - codes[::-1]).astype(np.uint8))


def test_topk_oracle_orders_ties_by_column():
    A = np.full((1, 16), 0x38, np.uint8)
    B = np.zeros((10, 16), np.uint8)
    B[[2, 5, 7]] = 0x38          # three columns tie at the top score
    v, l = orc.topk_e4m3(A, B, 4, 1)
    assert list(l[0]) == [3, 6, 8, 1] and list(v[0]) == [16.0, 16.0, 16.0, 0.0]


# ------------------------------------------------ the reference's own experiment outputs
# RotorMap/experiments/rope_{mutation,double_mutation,shift_mutation}_sweep.jl
# ran the reference's fp64 encoder (k = 20,000, s5 m1 c5, normalize 0) on
# Julia-seeded fixtures and committed their curves;
# tests/golden/make_sweep_golden.py copies them into rope_sweeps.json.
# rotormap.jlrandom draws the same fixtures (Julia's Xoshiro stream, the
# reference's generate_reference / mutate / mutate_shift), so the oracle is
# compared with the reference's own float64 results value for value.

SWEEPS = json.loads((Path(__file__).parent / "golden" / "rope_sweeps.json").read_text())
SK, SS, SM, SC = 20000, 5, 1, 5
# the curves are float64 results of the same arithmetic; 1e-12 absolute is
# ~5,000 ulp at these magnitudes, while a fixture that differs in a single
# base moves an inner product by ~1e-4
PIN_ATOL = 1e-12


def _pack(codes_list):
    from rotormap import synth
    return synth.pack_reads(codes_list, SK)


def _ip(e0, e1):
    """(Re<z0,z1>, |<z0,z1>|) of two split [Re; Im] unit vectors
    (rope_inner, RotorMap/experiments/rope_mutation_sweep.jl:67-73)."""
    D = e0.size // 2
    re_ = float(e0 @ e1)
    im = float(e0[:D] @ e1[D:] - e0[D:] @ e1[:D])
    return re_, math.hypot(re_, im)


def _fragment():
    from rotormap import jlrandom
    f = SWEEPS["fragment"]
    return jlrandom.generate_reference(f["n"], f["seed"])


def _pre(frag, name):
    from rotormap import jlrandom
    pre = SWEEPS["sweeps"][name]["pre"]
    if pre is None:
        return frag
    rng = jlrandom.Xoshiro(pre["seed"])
    if pre["kind"] == "mutate":
        return jlrandom.mutate(frag, pre["err"], rng)
    return jlrandom.mutate_shift(frag, pre["err"], rng)


def _check_rows(name, stride):
    from rotormap import jlrandom
    frag = _fragment()
    pre = _pre(frag, name)
    rows = SWEEPS["sweeps"][name]["rows"]
    rows = rows[::stride] + ([rows[-1]] if (len(rows) - 1) % stride else [])
    base = SWEEPS["copy_seed_base"]
    muts = [frag] + [jlrandom.mutate(pre, err, jlrandom.Xoshiro(base + i)) for i, err, _, _ in rows]
    assert all(m.size == SK for m in muts)
    e, _ = orc.rope_f64(_pack(muts), SK, SS, SM, SC)
    worst = 0.0
    for j, (i, err, ip_re, ip_abs) in enumerate(rows):
        got = _ip(e[0], e[j + 1])
        worst = max(worst, abs(got[0] - ip_re), abs(got[1] - ip_abs))
    assert worst < PIN_ATOL, f"{name} sweep: largest difference {worst:.3e}"
    return len(rows)


def test_julia_stream_restatement():
    """Julia's Xoshiro draws as the reference's fixtures use them: the
    shift sweep's pre-mutation draws its 500-base tail from Xoshiro(42), the
    generator that made the fragment, so the tail is the fragment's own head
    and the shifted copy is a rotation."""
    from rotormap import jlrandom
    frag = _fragment()
    assert frag.size == SK and set(np.unique(frag)) <= {0, 1, 2, 3}
    assert np.array_equal(jlrandom.mutate_shift(frag, 0.05, jlrandom.Xoshiro(42)), np.roll(frag, -500))
    # mutate keeps the length; err = 0 is the identity
    assert np.array_equal(jlrandom.mutate(frag, 0.0, jlrandom.Xoshiro(43)), frag)
    m = jlrandom.mutate(frag, 0.25, jlrandom.Xoshiro(7))
    assert m.size == SK and 0.4 < float(np.mean(m != frag)) < 0.9
    # the error grid of the sweeps
    errs = [r[1] for r in SWEEPS["sweeps"]["mutation"]["rows"]]
    assert np.array_equal(np.array(errs), jlrandom.sweep_errs(1000))


def test_generate_reads_follows_the_reference_self_test():
    """The reference self-test's stage A on Julia-exact draws
    (RotorMap/selftest.jl:106-134): generate_reference(50_000; seed = 1);
    generate_reads at err = 0 gives exact windows at 0-based starts in
    0..N-k; mutate at err = 0 is the identity, and at err = 0.05 keeps the
    length, changes bases and is deterministic in its generator."""
    from rotormap import jlrandom
    ref = jlrandom.generate_reference(50_000, 1)
    assert ref.size == 50_000 and ref.max() <= 3
    reads, pos = jlrandom.generate_reads(ref, 1_000, 64, err=0.0, seed=2)
    assert len(reads) == 64 and pos.min() >= 0 and pos.max() <= 50_000 - 1_000
    assert all(np.array_equal(r, ref[p:p + 1_000]) for r, p in zip(reads, pos))
    assert np.array_equal(jlrandom.mutate(ref, 0.0, jlrandom.Xoshiro(3)), ref)
    m1 = jlrandom.mutate(ref, 0.05, jlrandom.Xoshiro(4))
    m2 = jlrandom.mutate(ref, 0.05, jlrandom.Xoshiro(4))
    m3 = jlrandom.mutate(ref, 0.05, jlrandom.Xoshiro(5))
    assert m1.size == ref.size and not np.array_equal(m1, ref)
    assert np.array_equal(m1, m2) and not np.array_equal(m1, m3)


def test_shift_anchor_of_the_reference_sweep():
    """The shift sweep's err = 0 row (fragment vs its 500-base shift) to
    within PIN_ATOL of the reference's float64 value."""
    row = SWEEPS["sweeps"]["shift"]["rows"][0]
    assert row[1] == 0.0
    frag = _fragment()
    e, _ = orc.rope_f64(_pack([frag, _pre(frag, "shift")]), SK, SS, SM, SC)
    got = _ip(e[0], e[1])
    assert abs(got[0] - row[2]) < PIN_ATOL and abs(got[1] - row[3]) < PIN_ATOL


def test_mutation_sweep_of_the_reference():
    """Every 8th row of the single-mutation sweep (and its last) equals the
    reference's float64 inner products."""
    assert _check_rows("mutation", 8) >= 125


def test_periodic_fragment_table_of_the_reference():
    """The legacy periodic-fragment table (RotorMap/legacy/test/ropeperiod.jl:
    a 4,002-base Xoshiro(42) motif tiled to k = 20,000, whose five copies
    nearly cancel -- the phases are tested where the encoding is dominated
    by a few hundred defect windows): all 51 rows within the table's printed
    precision (6 decimals)."""
    from rotormap import jlrandom
    per = SWEEPS["periodic"]
    frag = jlrandom.periodic_fragment(per["k"], per["period"], per["seed"])
    rows = per["rows"]
    muts = [frag] + [jlrandom.mutate(frag, err, jlrandom.Xoshiro(per["seed"] + i)) for i, err, _, _ in rows if i > 0]
    e, _ = orc.rope_f64(_pack(muts), SK, SS, SM, SC)
    got = [(1.0, 1.0)] + [_ip(e[0], x) for x in e[1:]]
    half_ulp6 = 0.5e-6 + 1e-12
    for (i, err, ip_re, ip_abs), g in zip(rows, got):
        assert abs(g[0] - ip_re) <= half_ulp6 and abs(g[1] - ip_abs) <= half_ulp6, (err, g, ip_re, ip_abs)
    assert abs(_ip(e[0], e[0])[0] - 1.0) < 1e-12


@pytest.mark.parametrize("name", ["double", "shift"])
def test_pre_mutated_sweeps_of_the_reference(name):
    """The double-mutation sweep (0.3 pre-mutation by mutate) and the shift
    sweep (0.05 pre-shift by mutate_shift): every other kept row equals the
    reference's float64 inner products."""
    assert _check_rows(name, 2) >= 50
