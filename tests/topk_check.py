"""Top-k row checks with ties made explicit.

The reference checks a top-k row as: sorted descending, the value multiset
equal to the exact top-k, every location > 0 and carrying its value
(`_assert_topk_rows`, RotorMap/search/engine_fp8.jl:757-769;
RotorMap/gemm/topk_kernels.jl:539-544).  Where scores are compared with a
tolerance (fp16 rounding steps, accumulation order), the same check reads:

  * the row is sorted descending and its locations are distinct, in 1..N;
  * its value at every rank is within `tol` of the oracle's value there;
  * every returned location's oracle score is within `tol` of the value the
    row carries for it -- so a location that differs from the oracle's at a
    rank is a tie within `tol` with the oracle's entry at that rank.

`assert_topk_rows` returns how many (row, rank) locations differ from the
oracle's, each of them shown to be such a tie.
"""
import numpy as np

from oracle import oracle as orc


def oracle_scores_at(a8, B, locs, mode=0, scaleA=None, scaleB=None):
    """The oracle's score (orc_scores_e4m3 arithmetic: fp64 dot, then the
    mode's rounding / column scale, then the row scale) of every (row,
    location) pair of locs (nb, k), 1-based; location 0 scores -inf."""
    a8 = np.ascontiguousarray(a8, np.uint8)
    nb, k = locs.shape
    out = np.full((nb, k), -np.inf, np.float32)
    for r in range(nb):
        cols = locs[r].astype(np.int64) - 1
        ok = cols >= 0
        if not ok.any():
            continue
        c = cols[ok]
        sb = None if scaleB is None else np.asarray(scaleB, np.float32)[c]
        sc = orc.scores_e4m3(a8[r], np.asarray(B)[c], mode, sb)
        if mode == 2 and scaleA is not None:
            sc = (sc * np.float32(scaleA[r])).astype(np.float32)
        out[r, ok] = sc
    return out


def assert_topk_rows(vals, locs, ref_vals, ref_locs, scores_at, tol, N=None):
    """See the module doc.  scores_at: (nb, k) oracle scores of `locs`."""
    vals, locs = np.asarray(vals), np.asarray(locs)
    ref_vals, ref_locs = np.asarray(ref_vals), np.asarray(ref_locs)
    assert vals.shape == ref_vals.shape and locs.shape == vals.shape
    assert np.all(np.diff(vals, axis=1) <= 0), "a row is not sorted descending"
    assert np.all(locs >= 1) and (N is None or np.all(locs <= N)), "location out of 1..N"
    for r in range(locs.shape[0]):
        assert np.unique(locs[r]).size == locs.shape[1], f"row {r}: repeated location"
    np.testing.assert_allclose(vals, ref_vals, rtol=0, atol=tol, err_msg="top-k values differ beyond tol")
    np.testing.assert_allclose(scores_at, vals, rtol=0, atol=tol,
                               err_msg="a returned location does not carry its value (within tol)")
    diff = locs != ref_locs
    # every differing location is a tie within tol with the oracle's entry
    # at that rank (implied by the two checks above; stated for the record)
    assert np.all(np.abs(scores_at[diff] - ref_vals[diff]) <= 2 * tol)
    return int(diff.sum())
