"""Generate tests/golden/rope_golden.json: closed-form rope embeddings of
periodic fragments.

For a fragment whose bases repeat with period P, window p's s-mer (and so its
scrambled c-mer bin) depends only on r = p mod P, and the phasor sum of one
residue class is a geometric series:

    sum_{j=0}^{n_r-1} exp(i*theta*(r + j*P)) = exp(i*theta*r) * (1 - w^n_r) / (1 - w),
    w = exp(i*theta*P)   (or n_r when w == 1).

The bins follow the reference's definitions (RotorMap/encode/reference.jl:37-
105): little-endian s-mer field, csmer = lower ^ ((upper * 0x9E3779B1) &
(4^c-1)), bin = csmer*m + idm, theta = factor*2*pi/k with factor = 1 (m = 1)
or 2*idm/(m-1)+1, the "GG..G" c-mer bin 2*sum_{i<c}4^i zeroed, normalize
mode 0 (divide by sqrt(sum |h|^2) + 1e-16), split [Re; Im] layout.  The values
are evaluated with Python integers and complex128 closed forms -- a derivation
independent of the summation loops of the oracle and of the GPU kernel.

Run: python tests/golden/make_golden.py   (rewrites the JSON next to it)
"""
import cmath
import json
import math
from pathlib import Path

CODE = {"A": 0, "C": 1, "G": 2, "T": 3}

CASES = [
    # (name, unit, k, s, m, c)
    ("all_A", "A", 150, 8, 4, 4),
    ("all_C", "C", 150, 8, 4, 4),
    ("all_G", "G", 150, 8, 4, 4),
    ("all_T", "T", 150, 8, 4, 4),
    ("AC", "AC", 150, 8, 4, 4),
    ("ACGT", "ACGT", 150, 8, 4, 4),
    ("AACCGGTT", "AACCGGTT", 150, 8, 4, 4),
    ("ACGTTGCA", "ACGTTGCA", 100, 8, 4, 4),
    ("GATTACA", "GATTACA", 37, 5, 1, 3),
    ("CAT", "CAT", 250, 8, 2, 3),
    ("TTAGGG", "TTAGGG", 2001, 5, 1, 4),
    ("GGGGGC", "GGGGGC", 150, 8, 4, 4),
]


def scramble(smer: int, c: int) -> int:
    cb = (1 << (2 * c)) - 1
    lower = smer & cb
    upper = smer >> (2 * c)
    return lower ^ (((upper * 0x9E3779B1) & 0xFFFFFFFF) & cb)


def fragment(unit: str, k: int):
    return [CODE[unit[j % len(unit)]] for j in range(k)]


def golden(unit, k, s, m, c):
    P = len(unit)
    codes = fragment(unit, k)
    nw = k - s + 1
    nbin = m * 4 ** c
    hist = [0j] * nbin
    for r in range(min(P, nw)):
        smer = sum(codes[r + j] << (2 * j) for j in range(s))
        cs = scramble(smer, c)
        n_r = (nw - 1 - r) // P + 1  # windows r, r+P, ... < nw
        for idm in range(m):
            f = 1.0 if m == 1 else 2.0 * idm / (m - 1) + 1.0
            th = f * (2.0 * math.pi / k)
            w = cmath.exp(1j * th * P)
            if abs(w - 1) < 1e-300:
                geo = n_r
            else:
                geo = (1 - w ** n_r) / (1 - w)
            hist[cs * m + idm] += cmath.exp(1j * th * r) * geo
    allones = sum(4 ** i for i in range(c))
    g = 2 * allones
    for idm in range(m):
        hist[g * m + idm] = 0j
    nrm = math.sqrt(sum(abs(h) ** 2 for h in hist)) + 1e-16
    nz = {b: [h.real / nrm, h.imag / nrm] for b, h in enumerate(hist) if h != 0}
    return nz, nrm


def main():
    out = []
    for name, unit, k, s, m, c in CASES:
        nz, nrm = golden(unit, k, s, m, c)
        out.append(dict(name=name, unit=unit, k=k, s=s, m=m, c=c, nbin=m * 4 ** c, norm=nrm,
                        bins={str(b): v for b, v in sorted(nz.items())}))
    p = Path(__file__).with_name("rope_golden.json")
    p.write_text(json.dumps(out, indent=1))
    print(f"wrote {p} ({len(out)} cases)")


if __name__ == "__main__":
    main()
