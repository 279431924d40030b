"""Summarise the reference's committed mutation-sweep curve into error-rate
bins: tests/golden/rope_mutation_sweep_bins.json.

Source: RotorMap/experiments/out/rope_mutation_sweep.csv in the reference
checkout (err, ip_re, ip_abs per mutated copy; written by
RotorMap/experiments/rope_mutation_sweep.jl: a random 20,000-base fragment,
the fp64 reference encoder at s=5 m=1 c=5, normalize=0, 1000 copies mutated
by RotorMap/common/dna.jl's `mutate` at err = 0.5*(i-1)/999).  The copies
come from Julia's Xoshiro and cannot be regenerated here, so the fixture
keeps per-bin statistics (count, mean, standard deviation of ip_re and
ip_abs) that a restatement with any RNG must reproduce within sampling
error.

The shift sweep's first row (RotorMap/experiments/out/
rope_shift_mutation_sweep.csv, err = 0: the pristine fragment against its
500-base shifted copy, same encoder) is kept verbatim as a second,
near-deterministic anchor.

Usage: python tests/golden/make_sweep_bins.py path/to/reference/checkout
"""
import csv
import json
import sys
from pathlib import Path

import numpy as np

NBINS = 20


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_sweep_bins.py path/to/reference/checkout")
    root = Path(sys.argv[1])
    src = root / "RotorMap" / "experiments" / "out" / "rope_mutation_sweep.csv"
    rows = list(csv.DictReader(open(src)))
    err = np.array([float(r["err"]) for r in rows])
    ipre = np.array([float(r["ip_re"]) for r in rows])
    ipabs = np.array([float(r["ip_abs"]) for r in rows])
    edges = np.linspace(0.0, 0.5, NBINS + 1)
    bins = []
    for b in range(NBINS):
        sel = (err >= edges[b]) & ((err < edges[b + 1]) if b + 1 < NBINS else (err <= edges[b + 1]))
        bins.append({"err_lo": float(edges[b]), "err_hi": float(edges[b + 1]), "count": int(sel.sum()),
                     "ip_re_mean": float(ipre[sel].mean()), "ip_re_std": float(ipre[sel].std(ddof=1)),
                     "ip_abs_mean": float(ipabs[sel].mean()), "ip_abs_std": float(ipabs[sel].std(ddof=1))})
    shift = next(csv.DictReader(open(root / "RotorMap" / "experiments" / "out" / "rope_shift_mutation_sweep.csv")))
    out = {"source": "RotorMap/experiments/out/rope_mutation_sweep.csv",
           "encoder": {"k": 20000, "s": 5, "m": 1, "c": 5, "normalize": 0},
           "points": len(rows), "bins": bins,
           "shift_anchor": {"source": "RotorMap/experiments/out/rope_shift_mutation_sweep.csv (err = 0 row)",
                            "shift": 500, "ip_re": float(shift["ip_re"]), "ip_abs": float(shift["ip_abs"])}}
    dst = Path(__file__).with_name("rope_mutation_sweep_bins.json")
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {dst} ({len(rows)} points, {NBINS} bins)")


if __name__ == "__main__":
    main()
