"""Julia-exact fixture draws: the reference's `generate_reference`,
`generate_reads`, `mutate` and `mutate_shift` (RotorMap/common/dna.jl) on
the same random stream as Julia's `Random` standard library.

The reference seeds every fixture with `Xoshiro(seed)` from Julia's
`Random` stdlib (julia_version 1.12.2 in RotorMap/Manifest.toml; the stdlib
is not vendored in the reference tree).  Its published algorithms, restated
here:

  * seeding: SHA-256 over the seed's 32-bit limbs, least significant first,
    each as 4 little-endian bytes; a negative seed is complemented first and
    the byte 0x01 is appended after its limbs.  The 32-byte digest, read as
    four little-endian UInt64, is the xoshiro256++ state (s0, s1, s2, s3);
  * `rand(rng, UInt64)`: one xoshiro256++ output
    (rotl(s0 + s3, 23) + s0, then the standard state update);
    `rand(rng, Int64)` is the same 64 bits as a signed integer;
  * `rand(rng, Float64)`: (u >>> 11) * 2^-53;
  * `rand(rng, collection)` of n elements, and `rand(rng, a:b)` of n
    values (`0x00:0x03` included): Lemire's nearly-divisionless method on a
    64-bit draw (64-bit product, the high word is the 0-based index, a low
    word below (2^64 - n) mod n is redrawn).

`mutate` goes through the reference's rope structure
(RotorMap/common/treearrays.jl) with its leaf size of 1,000, so the edits
land where the reference's land, including its routing of a node's
deletions that all fall in the left half: `deleteat!` hands them to the
RIGHT child at the same offsets (treearrays.jl:152-153).

These draws reproduce the reference's committed sweep curves
(RotorMap/experiments/out/rope_*_sweep.csv) value for value, and the
periodic-fragment table of RotorMap/legacy/test/ropeperiod.jl to its
printed 6 decimals; they are fixture generators, not part of the mapping
path.
"""
from __future__ import annotations

import hashlib
import math
import struct

import numpy as np

_M64 = (1 << 64) - 1


def _rotl(x: int, k: int) -> int:
    return ((x << k) | (x >> (64 - k))) & _M64


def hash_seed(seed: int) -> tuple:
    """The xoshiro256++ state Julia's `Xoshiro(seed)` starts from."""
    seed = int(seed)
    neg = seed < 0
    if neg:
        seed = ~seed
    data = b""
    while True:
        data += struct.pack("<I", seed & 0xFFFFFFFF)
        seed >>= 32
        if seed == 0:
            break
    if neg:
        data += b"\x01"
    return struct.unpack("<4Q", hashlib.sha256(data).digest())


class Xoshiro:
    """Julia's `Random.Xoshiro` (xoshiro256++) with the draws the reference's
    fixtures use."""

    def __init__(self, seed: int):
        self.s = list(hash_seed(seed))

    def rand_u64(self) -> int:
        s0, s1, s2, s3 = self.s
        res = (_rotl((s0 + s3) & _M64, 23) + s0) & _M64
        t = (s1 << 17) & _M64
        s2 ^= s0
        s3 ^= s1
        s1 ^= s2
        s0 ^= s3
        s2 ^= t
        s3 = _rotl(s3, 45)
        self.s = [s0, s1, s2, s3]
        return res

    def rand_i64(self) -> int:
        x = self.rand_u64()
        return x - (1 << 64) if x >> 63 else x

    def rand_f64(self) -> float:
        return float(self.rand_u64() >> 11) * 2.0 ** -53

    def rand_index(self, n: int) -> int:
        """0-based index of `rand(rng, c)` for a collection of n elements."""
        thresh = ((1 << 64) - n) % n
        while True:
            m = self.rand_u64() * n
            if (m & _M64) >= thresh:
                return m >> 64


def generate_reference(n: int, seed: int) -> np.ndarray:
    """`generate_reference(N; seed)` (RotorMap/common/dna.jl:85-94): N bases
    (codes 0..3) drawn by `rand(Xoshiro(seed), UInt8.(0:3), N)`."""
    rng = Xoshiro(seed)
    return np.array([rng.rand_index(4) for _ in range(int(n))], np.uint8)


class _Rope:
    """The reference's TreeArray (RotorMap/common/treearrays.jl:19-40):
    halves split at n÷2 down to leaves of at most `mll` elements; indices
    1-based as there."""

    __slots__ = ("length", "leaf", "data", "left", "right")

    def __init__(self, data, mll: int):
        n = len(data)
        self.length = n
        if n <= mll:
            self.leaf, self.data, self.left, self.right = True, list(data), None, None
        else:
            n2 = n // 2
            self.leaf, self.data = False, None
            self.left, self.right = _Rope(data[:n2], mll), _Rope(data[n2:], mll)

    def _split(self, inds):
        nl = self.left.length
        m2 = 0
        while m2 < len(inds) and inds[m2] <= nl:  # inds sorted: searchsorted(inds, nleft).stop
            m2 += 1
        return nl, m2

    def subsat(self, inds, vals):
        """subsat! (treearrays.jl:100-135)."""
        if self.leaf:
            for i, v in zip(inds, vals):
                self.data[i - 1] = v
            return
        nl, m2 = self._split(inds)
        if m2 < len(inds):
            self.right.subsat([i - nl for i in inds[m2:]], vals[m2:])
        if m2 > 0:
            self.left.subsat(inds[:m2], vals[:m2])

    def deleteat(self, inds):
        """deleteat! (treearrays.jl:137-171), including its routing of an
        all-left set of deletions to the right child."""
        self.length -= len(inds)
        if self.leaf:
            if inds and (inds[0] < 1 or inds[-1] > len(self.data)):
                raise IndexError("deletion outside the leaf (BoundsError in the reference)")
            drop = set(i - 1 for i in inds)
            self.data = [v for j, v in enumerate(self.data) if j not in drop]
            return
        nl, m2 = self._split(inds)
        if m2 == len(inds):
            self.right.deleteat(list(inds))
        elif m2 == 0:
            self.right.deleteat([i - nl for i in inds])
        else:
            self.right.deleteat([i - nl for i in inds[m2:]])
            self.left.deleteat(inds[:m2])

    def insertat(self, inds, vals):
        """insertat! (treearrays.jl:173-220): a leaf inserts from the last
        index down, so every index refers to the sequence before the
        insertions."""
        self.length += len(inds)
        if self.leaf:
            for i in range(len(inds) - 1, -1, -1):
                self.data.insert(inds[i] - 1, vals[i])
            return
        nl, m2 = self._split(inds)
        if m2 < len(inds):
            self.right.insertat([i - nl for i in inds[m2:]], vals[m2:])
        if m2 > 0:
            self.left.insertat(inds[:m2], vals[:m2])

    def flatten(self, out):
        if self.leaf:
            out.extend(self.data)
        else:
            self.left.flatten(out)
            self.right.flatten(out)
        return out


def mutate(dna, err: float, rng: Xoshiro, mll: int = 1000) -> np.ndarray:
    """`mutate(dna, err; rng, mll)` (RotorMap/common/dna.jl:120-183):
    n_err = ceil(n*err) edits, n_ins = n_del = floor(n_err/3), the rest
    substitutions; four child generators seeded by `rand(rng, Int64)` draw
    the substitution positions and letters, the deletion positions and the
    insertion positions and letters; the rope applies substitutions, then
    deletions, then insertions.  Returns the mutated codes."""
    dna = np.asarray(dna, np.uint8)
    n = int(dna.size)
    n_err = int(math.ceil(n * err))
    n_ins = int(math.floor(n_err * (1 / 3)))
    n_del = n_ins
    n_sub = n_err - n_ins - n_del
    rngs = [Xoshiro(rng.rand_i64()) for _ in range(4)]
    inds_s = sorted(int(math.ceil(n * rngs[0].rand_f64())) for _ in range(n_sub))
    # rand(rngs[1], [1, 2, 3]) added to the original letter, mod 4
    vals_s = [(int(dna[inds_s[i] - 1]) + 1 + rngs[0].rand_index(3)) % 4 for i in range(n_sub)]
    inds_d = sorted(int(math.ceil((n - t) * rngs[1].rand_f64())) for t in range(n_del))
    for i in range(1, n_del):
        inds_d[i] = max(inds_d[i], inds_d[i - 1] + 1)
    inds_i = sorted(int(math.ceil((n - n_del) * rngs[2].rand_f64())) for _ in range(n_ins))
    vals_i = [rngs[3].rand_index(4) for _ in range(n_ins)]
    rope = _Rope(dna.tolist(), mll)
    rope.subsat(inds_s, vals_s)
    rope.deleteat(inds_d)
    rope.insertat(inds_i, vals_i)
    return np.array(rope.flatten([]), np.uint8)


def mutate_shift(dna, err: float, rng: Xoshiro, shift: int | None = None) -> np.ndarray:
    """`mutate_shift(dna, err; shift, rng)` (RotorMap/common/dna.jl:185-195):
    drop the first floor(n*err/2) bases and append as many drawn bases."""
    dna = np.asarray(dna, np.uint8)
    n = int(dna.size)
    if shift is None:
        shift = int(math.floor(n * err / 2))
    tail = np.array([rng.rand_index(4) for _ in range(shift)], np.uint8)
    return np.concatenate([dna[shift:], tail])


def generate_reads(dna_ref, k: int, n: int = 1, err: float = 0.15, seed: int = 0):
    """`generate_reads(dna_ref, k, n; err, seed)` (RotorMap/common/dna.jl:
    96-118): n 0-based window starts drawn by `rand(rng, 0:N-k, n)` from
    `Xoshiro(seed)`, then one child generator per read seeded by
    `rand(rng, Int64)`, and each read `mutate(window, err; rng = child)`.
    Returns (reads, starts)."""
    dna_ref = np.asarray(dna_ref, np.uint8)
    N = int(dna_ref.size)
    if k > N:
        raise ValueError(f"k = {k} exceeds the reference length {N}")
    rng = Xoshiro(seed)
    pos = [rng.rand_index(N - k + 1) for _ in range(int(n))]
    kids = [Xoshiro(rng.rand_i64()) for _ in range(int(n))]
    reads = [mutate(dna_ref[p:p + k], err, kids[i]) for i, p in enumerate(pos)]
    return reads, np.array(pos, np.int64)


def periodic_fragment(k: int, period: int, seed: int) -> np.ndarray:
    """`periodic_fragment(k, p, seed)` (RotorMap/legacy/test/ropeperiod.jl):
    a motif of `period` bases drawn by `rand(Xoshiro(seed), 0x00:0x03)`,
    tiled to exactly k bases."""
    rng = Xoshiro(seed)
    motif = np.array([rng.rand_index(4) for _ in range(int(period))], np.uint8)
    return motif[np.arange(int(k)) % int(period)]


def sweep_errs(npts: int = 1000) -> np.ndarray:
    """The sweeps' error grid `range(0.0, 0.5; length = npts)`."""
    return np.array([0.5 * i / (npts - 1) for i in range(npts)])
