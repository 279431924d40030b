"""Copy the reference's committed encoder sweep curves into
tests/golden/rope_sweeps.json.

Sources, in a reference checkout (RotorMap/experiments/out/):
  * rope_mutation_sweep.csv -- written by
    RotorMap/experiments/rope_mutation_sweep.jl: fragment
    generate_reference(20_000; seed = 42), the fp64 encoder
    `_ref_rope_frag_real` at s=5 m=1 c=5 normalize=0, copy i (1-based)
    = mutate(fragment, err_i; rng = Xoshiro(42 + i)), err_i = 0.5(i-1)/999;
    columns err, Re<z0, zi>, |<z0, zi>|;
  * rope_double_mutation_sweep.csv -- the same sweep applied on top of
    pre = mutate(fragment, 0.3; rng = Xoshiro(42))
    (RotorMap/experiments/rope_double_mutation_sweep.jl);
  * rope_shift_mutation_sweep.csv -- the same sweep on top of
    pre = mutate_shift(fragment, 0.05; rng = Xoshiro(42))
    (RotorMap/experiments/rope_shift_mutation_sweep.jl).

Every row of the single sweep is kept; every 10th row and the last of the
other two.  Values are the CSVs' own decimal strings parsed as float64
(Julia prints the shortest round-trip form, so they are the reference's
exact float64 results).

Also the RESULTS table of RotorMap/legacy/test/ropeperiod.jl (written in
that file's header comment, 6 decimals): a 4,002-base motif drawn by
`rand(Xoshiro(42), 0x00:0x03)` tiled to k = 20,000, the same fp64 encoder,
copy i = mutate(fragment, 0.01 i; rng = Xoshiro(42 + i)), i = 1..50, plus
the err = 0 row.

Usage: python tests/golden/make_sweep_golden.py path/to/reference/checkout
"""
import csv
import json
import re
import sys
from pathlib import Path

SWEEPS = {
    "mutation": {"csv": "rope_mutation_sweep.csv", "pre": None, "stride": 1},
    "double": {"csv": "rope_double_mutation_sweep.csv", "pre": {"kind": "mutate", "err": 0.3, "seed": 42},
               "stride": 10},
    "shift": {"csv": "rope_shift_mutation_sweep.csv", "pre": {"kind": "mutate_shift", "err": 0.05, "seed": 42},
              "stride": 10},
}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_sweep_golden.py path/to/reference/checkout")
    out_dir = Path(sys.argv[1]) / "RotorMap" / "experiments" / "out"
    out = {"encoder": {"k": 20000, "s": 5, "m": 1, "c": 5, "normalize": 0},
           "fragment": {"n": 20000, "seed": 42}, "copy_seed_base": 42, "sweeps": {}}
    for name, spec in SWEEPS.items():
        rows = list(csv.DictReader(open(out_dir / spec["csv"])))
        keep = sorted(set(range(0, len(rows), spec["stride"])) | {len(rows) - 1})
        out["sweeps"][name] = {
            "source": f"RotorMap/experiments/out/{spec['csv']}",
            "pre": spec["pre"], "points": len(rows),
            "rows": [[i + 1, float(rows[i]["err"]), float(rows[i]["ip_re"]), float(rows[i]["ip_abs"])]
                     for i in keep],
        }
    # the legacy periodic-fragment table: "err Re<IP> |IP|" rows, two per line
    table = {}
    pat = re.compile(r"#\s+(0\.\d\d)\s+(-?\d\.\d+)\s+(\d\.\d+)(?:\s+(0\.\d\d)\s+(-?\d\.\d+)\s+(\d\.\d+))?\s*$")
    for line in open(Path(sys.argv[1]) / "RotorMap" / "legacy" / "test" / "ropeperiod.jl"):
        m = pat.match(line)
        if m:
            for g in (1, 4):
                if m.group(g):
                    table[m.group(g)] = [float(m.group(g + 1)), float(m.group(g + 2))]
    out["periodic"] = {"source": "RotorMap/legacy/test/ropeperiod.jl (RESULTS comment)", "k": 20000, "period": 4002,
                       "seed": 42, "decimals": 6,
                       "rows": [[int(round(float(e) * 100)), float(e), v[0], v[1]] for e, v in sorted(table.items())]}
    dst = Path(__file__).with_name("rope_sweeps.json")
    dst.write_text(json.dumps(out, separators=(",", ":")) + "\n")
    print(f"wrote {dst} ({sum(len(s['rows']) for s in out['sweeps'].values())} sweep rows, "
          f"{len(out['periodic']['rows'])} periodic rows)")


if __name__ == "__main__":
    main()
