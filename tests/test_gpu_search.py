"""GPU parity of the fused fp8 GEMM + top-k engine against the oracle's
brute-force scores (the reference's checks: test_seg_rowtopk_merge_kernel,
RotorMap/gemm/topk_kernels.jl:518-552, and _check_engine_gemm_topk,
RotorMap/search/engine_fp8.jl:777-834)."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc

import rotormap as rm

pytestmark = pytest.mark.gpu

E4M3_INT = {0: 0x00, 1: 0x38, 2: 0x40, 3: 0x44, -1: 0xB8, -2: 0xC0, -3: 0xC4}


def int_e4m3(rng, shape, lo=-3, hi=3):
    """e4m3 bytes of small integers: every dot product is an exact small
    integer in any summation order, so scores, ties and tie order are exact."""
    v = rng.integers(lo, hi + 1, size=shape)
    lut = np.zeros(7, np.uint8)
    for x, b in E4M3_INT.items():
        lut[x + 3] = b
    return lut[v + 3], v


def unit_e4m3(rng, n, rdim):
    x = rng.standard_normal((n, rdim)).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    return orc.quantize_parity(x)


def run_engine(A8, B8, k, score="f16", scaleA=None, scaleB=None, splits=0, ctas=0, kernel="auto"):
    B = torch.from_numpy(B8).cuda()
    A = torch.from_numpy(A8).cuda()
    sb = torch.from_numpy(scaleB).cuda() if scaleB is not None else None
    sa = torch.from_numpy(scaleA).cuda() if scaleA is not None else None
    eng = rm.TopKEngine(B, k=k, rows_cap=A8.shape[0], score=score, scaleB=sb, splits=splits, ctas=ctas,
                        kernel=kernel)
    v, l = eng.search(A, A8.shape[0], sa)
    torch.cuda.synchronize()
    from rotormap._lib import check, lib
    check(lib().r2m_check_device_error(None))
    eng.close()
    return v.cpu().numpy(), l.cpu().numpy()


# the reference's top-k unit-test shapes (M, N) plus tile-edge cases
SHAPES = [(64, 100), (257, 128), (1000, 333), (1, 4096), (511, 2048), (2048, 16384), (33, 37),
          (64, 25), (64, 20), (129, 257), (128, 256), (300, 70001)]


@pytest.mark.parametrize("nb,N", SHAPES)
@pytest.mark.parametrize("score", ["f16", "f32"])
@pytest.mark.parametrize("kernel", ["1sm", "2sm"])
def test_topk_exact_integer_scores(nb, N, score, kernel):
    rng = np.random.default_rng(nb * 7 + N)
    rdim = 256
    A8, _ = int_e4m3(rng, (nb, rdim), -1, 1)
    B8, _ = int_e4m3(rng, (N, rdim), -1, 1)
    k = 20
    v, l = run_engine(A8, B8, k, score, kernel=kernel)
    ov, ol = orc.topk_e4m3(A8, B8, k, 0 if score == "f16" else 1)
    assert np.array_equal(v, ov)
    assert np.array_equal(l, ol)  # ties broken by ascending column, exactly


@pytest.mark.parametrize("k", [1, 5, 8, 16, 20, 32, 64])
def test_topk_k_values(k):
    rng = np.random.default_rng(k)
    A8, _ = int_e4m3(rng, (200, 128))
    B8, _ = int_e4m3(rng, (5000, 128))
    v, l = run_engine(A8, B8, k)
    ov, ol = orc.topk_e4m3(A8, B8, k, 0)
    assert np.array_equal(v, ov) and np.array_equal(l, ol)


@pytest.mark.parametrize("splits,ctas", [(1, 2), (3, 2), (7, 6), (0, 4), (128, 0)])
@pytest.mark.parametrize("kernel", ["1sm", "2sm"])
def test_topk_schedules(splits, ctas, kernel):
    """Forced column splits / few CTAs: several work units per CTA (pair)
    reuse the TMEM double buffer across units."""
    rng = np.random.default_rng(splits + 10 * ctas)
    A8, _ = int_e4m3(rng, (300, 256))
    B8, _ = int_e4m3(rng, (9000, 256))
    v, l = run_engine(A8, B8, 20, splits=splits, ctas=ctas, kernel=kernel)
    ov, ol = orc.topk_e4m3(A8, B8, 20, 0)
    assert np.array_equal(v, ov) and np.array_equal(l, ol)


@pytest.mark.parametrize("rdim", [16, 48, 128, 384, 2048])
@pytest.mark.parametrize("kernel", ["1sm", "2sm"])
def test_topk_rdim_tails(rdim, kernel):
    rng = np.random.default_rng(rdim)
    A8, _ = int_e4m3(rng, (300, rdim), -1, 1)
    B8, _ = int_e4m3(rng, (3000, rdim), -1, 1)
    v, l = run_engine(A8, B8, 20, "f32", kernel=kernel)
    ov, ol = orc.topk_e4m3(A8, B8, 20, 1)
    assert np.array_equal(v, ov) and np.array_equal(l, ol)


@pytest.mark.parametrize("score", ["f16", "f32", "scaled"])
def test_topk_realistic_values_within_tolerance(score):
    """Unit-norm rows quantised like the reference: the device accumulates in
    fp32 in its own order, so scores may differ from the exact oracle by fp32
    rounding (and, for f16, by one fp16 step at a rounding boundary)."""
    rng = np.random.default_rng(11)
    nb, N, rdim, k = 400, 20000, 2048, 20
    A8 = unit_e4m3(rng, nb, rdim)
    B8 = unit_e4m3(rng, N, rdim)
    sa = sb = None
    if score == "scaled":
        sa = rng.uniform(0.5, 2.0, nb).astype(np.float32)
        sb = rng.uniform(0.5, 2.0, N).astype(np.float32)
    mode = {"f16": 0, "f32": 1, "scaled": 2}[score]
    v, l = run_engine(A8, B8, k, score, sa, sb)
    ov, ol = orc.topk_e4m3(A8, B8, k, mode, sa, sb)
    tol = 1e-3 if score == "f16" else 2e-5
    assert np.all(np.diff(v, axis=1) <= 0)
    np.testing.assert_allclose(v, ov, atol=tol, rtol=0)
    # every returned location carries its value, and the sets agree up to ties
    for r in range(0, nb, 37):
        sc = orc.scores_e4m3(A8[r], B8, mode, sb)
        if score == "scaled":
            sc = sc * sa[r]
        np.testing.assert_allclose(sc[l[r] - 1], v[r], atol=tol, rtol=0)
        kth = ov[r, -1]
        assert np.all(sc[l[r] - 1] >= kth - 2 * tol)
        strict = set(np.flatnonzero(sc > kth + 2 * tol) + 1)
        assert strict <= set(l[r])


def test_engine_rejects_bad_arguments():
    B = torch.zeros((100, 64), dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError):
        rm.TopKEngine(B, k=101)
    with pytest.raises(rm.R2MError):
        from rotormap._lib import lib, check
        import ctypes
        h = ctypes.c_void_p()
        check(lib().r2m_engine_create(B.data_ptr(), None, 60, 100, 20, 10, 0, None, ctypes.byref(h)))
    eng = rm.TopKEngine(B, k=20, rows_cap=8)
    A = torch.zeros((9, 64), dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError):
        eng.search(A)


@pytest.mark.parametrize("score", ["f16", "scaled"])
@pytest.mark.parametrize("kernel", ["1sm", "2sm"])
def test_pair_kernel_epilogue_forms_agree(score, kernel):
    """Both kernels drain tiles with 8 epilogue warps (two column halves, two
    partial lists per row) when a work unit spans at most 8192 column tiles
    and with 4 warps otherwise; both forms give the same values, locations
    and tie order.  One split over 8,600 tiles takes the 4-warp form, two
    splits the 8-warp form."""
    rng = np.random.default_rng(77)
    nb, N, rdim = 300, 2_201_000, 16
    A8, _ = int_e4m3(rng, (nb, rdim), -1, 1)
    B8, _ = int_e4m3(rng, (N, rdim), -1, 1)
    sa = rng.uniform(0.5, 2.0, nb).astype(np.float32) if score == "scaled" else None
    sb = rng.uniform(0.5, 2.0, N).astype(np.float32) if score == "scaled" else None
    v1, l1 = run_engine(A8, B8, 20, score, sa, sb, splits=1, kernel=kernel)
    v2, l2 = run_engine(A8, B8, 20, score, sa, sb, splits=2, kernel=kernel)
    assert np.array_equal(v1, v2) and np.array_equal(l1, l2)
    # spot-check against brute-force scores of a few rows
    from oracle import oracle as orc
    for r in (0, 151, 299):
        # ranks follow the score before the per-row factor (a positive scale)
        sc = orc.scores_e4m3(A8[r], B8, 2 if score == "scaled" else 0, sb)
        order = np.lexsort((np.arange(N), -sc))[:20]
        assert list(l1[r]) == list(order + 1)


@pytest.mark.parametrize("k", [8, 20, 32, 64])
@pytest.mark.parametrize("kernel", ["1sm", "2sm"])
def test_pair_kernel_forced_epilogue_forms(k, kernel):
    """Forcing 4 or 8 epilogue warps (k = 64 always runs 4) changes nothing
    in the results, across split counts."""
    rng = np.random.default_rng(k)
    nb, N, rdim = 513, 70_001, 128
    A8, _ = int_e4m3(rng, (nb, rdim), -1, 1)
    B8, _ = int_e4m3(rng, (N, rdim), -1, 1)
    A = torch.from_numpy(A8).cuda()
    eng = rm.TopKEngine(torch.from_numpy(B8).cuda(), k=k, rows_cap=nb, kernel=kernel)
    ref = None
    for ep in ("4", "8", "auto"):
        for s in (1, 3, 17):
            eng.set_tuning(splits=s, epilogue=ep)
            v, l = eng.search(A, nb)
            out = (v.cpu().numpy(), l.cpu().numpy())
            if ref is None:
                ref = out
            assert np.array_equal(out[0], ref[0]) and np.array_equal(out[1], ref[1])
    with pytest.raises(ValueError):
        eng.set_tuning(epilogue="6")
    eng.close()


@pytest.mark.parametrize("epilogue", ["4", "8"])
@pytest.mark.parametrize("score", ["f16", "scaled"])
def test_pair_pacing_changes_only_the_schedule(epilogue, score):
    """Pair pacing (tuning reserved[3]) delays pairs but computes nothing
    differently: unpaced, the default window, the tightest window (1 tile)
    and a window wider than the index give identical values, locations and
    tie order, search after search, equal to the oracle."""
    rng = np.random.default_rng(41)
    nb, N, rdim = 600, 200_001, 128  # 3 pair read tiles x 782 column tiles
    A8, _ = int_e4m3(rng, (nb, rdim), -1, 1)
    B8, _ = int_e4m3(rng, (N, rdim), -1, 1)
    sa = rng.uniform(0.5, 2.0, nb).astype(np.float32) if score == "scaled" else None
    sb = rng.uniform(0.5, 2.0, N).astype(np.float32) if score == "scaled" else None
    B = torch.from_numpy(B8).cuda()
    A = torch.from_numpy(A8).cuda()
    sbt = torch.from_numpy(sb).cuda() if sb is not None else None
    sat = torch.from_numpy(sa).cuda() if sa is not None else None
    eng = rm.TopKEngine(B, k=20, rows_cap=nb, score=score, scaleB=sbt, kernel="2sm", epilogue=epilogue)
    outs = []
    for pace in (-1, 0, 1, 1 << 20, 0):
        eng.set_tuning(kernel="2sm", epilogue=epilogue, pace=pace)
        v, l = eng.search(A, nb, sat)
        torch.cuda.synchronize()
        outs.append((v.cpu().numpy(), l.cpu().numpy()))
    from rotormap._lib import check, lib
    check(lib().r2m_check_device_error(None))
    eng.close()
    rv, rl = orc.topk_e4m3(A8, B8, 20, 2 if score == "scaled" else 0, sa, sb)
    for v, l in outs:
        assert np.array_equal(v, rv) and np.array_equal(l, rl)


@pytest.mark.parametrize("nb,N", [(300, 70001), (64, 1000), (257, 4133)])
@pytest.mark.parametrize("k", [20, 32, 64])
@pytest.mark.parametrize("kernel", ["1sm", "2sm"])
def test_scaled_scores_exact_with_zero_and_negative_scales(nb, N, k, kernel):
    """Scaled scores with power-of-two row and column scales are exact, so
    the lists must equal the oracle's bit for bit, ties included, with zero
    column scales, negative column scales, a 32-column run of zero scales and
    a ragged last tile; k = 32 and 64 take the one-chunk-at-a-time and the
    64-entry reservoir epilogues."""
    rng = np.random.default_rng(nb + 3 * N + k)
    rdim = 256
    A8, _ = int_e4m3(rng, (nb, rdim), -2, 2)
    B8, _ = int_e4m3(rng, (N, rdim), -2, 2)
    sa = rng.choice(np.array([0.5, 1.0, 2.0], np.float32), nb)
    sb = rng.choice(np.array([0.25, 0.5, 1.0, 2.0, 4.0], np.float32), N)
    sb[rng.random(N) < 0.05] = 0.0
    sb[rng.random(N) < 0.02] *= -1.0
    sb[64:96] = 0.0  # one chunk of zero scales
    v, l = run_engine(A8, B8, k, "scaled", scaleA=sa, scaleB=sb, kernel=kernel)
    ov, ol = orc.topk_e4m3(A8, B8, k, 2, sa, sb)
    assert np.array_equal(v, ov)
    assert np.array_equal(l, ol)
