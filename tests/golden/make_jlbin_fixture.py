"""Hand-assembled index .bin fixture (tests/golden/index_tiny.bin).

The bytes below are written tag by tag, from the Julia Serialization stream
layout of the NamedTuple that the reference saves (RotorMap/index/build.jl:
755-768 via `serialize`, RotorMap/common/dna.jl:23-27), without using the
library's writer, so that the reader is checked against an independent
statement of the format and the writer against the same bytes.

Tags are positions in Julia's Serialization TAGS table (1-based):
  1 SYMBOL, 8 Int64 (type), 11 UInt128, 13 Float32 (type), 16 DATATYPE,
  20 TUPLE, 21 ARRAY, 31 MODULE, 33 STRING / String (type), 44 SHORTBACKREF,
  49 SHORTINT64, 52 OBJECT, 55 HEADER, 57 SHARED_REF, 68 (), 69 Bool (type),
  77 true, 78 nothing, symbols :Array 80, :Tuple 83, :c 104, :k 112, :m 114,
  :s 120, :Core 155; Int64 literals 0..32 are 223..255.
Objects that take a back-reference id, in stream order: the NamedTuple type
(0), :NamedTuple (1), :normalize (2), the Tuple type (3), Array{F8,2} (4),
the Float8_E4M3FN type (5), :Float8_E4M3FN (6), :DLFP8Types (7),
Array{Float32,2} (8), Array{String,1} (9), Array{Int64,1} (10),
Array{UInt8,1} (11), then the values: "indexreal.fp8.v1" (12),
"/data/tiny.fa" (13), embeds8 (14), norms (15), heads (16),
">chrA tiny" (17), starts (18), strand (19).

Run: python tests/golden/make_jlbin_fixture.py  (rewrites index_tiny.bin)
"""
import struct
from pathlib import Path

HERE = Path(__file__).resolve().parent

# the NamedTuple's values: 2 windows (n_frag 2 -> 4 columns), rdim 2*m*4^c
# with m = 1, c = 1 -> 8 bytes per column
K, KSTEP, S, M, C = 20, 2, 3, 1, 1
RDIM, N = 2 * M * 4 ** C, 4
EMBEDS8 = bytes(range(1, RDIM * N + 1))            # column j = bytes 8j+1 .. 8j+8
NORMS = [1.0, 1.0, 0.5, 2.0]                       # (m, N) = (1, 4)
HEADS = [">chrA tiny", ">chrA tiny", ">chrA tiny", ">B"]
STARTS = [1, 3, 1, 3]
STRAND = [0, 0, 1, 1]
SOURCE = "/data/tiny.fa"
FORMAT = "indexreal.fp8.v1"
# DLFP8Types' UUID (RotorMap/Manifest.toml:341) as a UInt128
UUID = 0xf4c16678_4a16_415b_82ef_ed337c5d6c7c


def sym(name):  # SYMBOL tag, u8 length, bytes
    b = name.encode()
    return bytes([1, len(b)]) + b


def string(s):  # STRING tag, u8 length, bytes
    b = s.encode()
    return bytes([33, len(b)]) + b


def i32(v):
    return struct.pack("<i", v)


CORE = bytes([31, 78, 155, 68])  # MODULE, nothing (no UUID), :Core, ()


def build() -> bytes:
    out = bytearray()
    out += bytes([55]) + b"JL" + bytes([20, 0x04, 0, 0, 0])   # HEADER, "JL", version 20, LE 64-bit
    out += bytes([52])                                          # OBJECT: a struct instance follows
    # type NamedTuple{names, Tuple{...}} (id 0)
    out += bytes([16]) + sym("NamedTuple")                      # DATATYPE, name (id 1)
    out += CORE + i32(2)                                        # module Core, 2 parameters
    names = ["format", "source", "k", "kstep", "s", "m", "c", "normalize", "fp8", "n_frag",
             "embeds8", "norms", "heads", "starts", "strand"]
    out += bytes([20, len(names)])                              # TUPLE of 15 symbols
    for nm in names:
        tag = {"k": 112, "s": 120, "m": 114, "c": 104}.get(nm)
        out += bytes([tag]) if tag else sym(nm)                 # :normalize takes id 2
    out += bytes([16, 83]) + CORE + i32(15)                     # Tuple{...} (id 3): DATATYPE, :Tuple
    out += bytes([0, 33]) * 2                                   # String, String
    out += bytes([0, 8]) * 6                                    # Int64 x 6 (k, kstep, s, m, c, normalize)
    out += bytes([69])                                          # Bool
    out += bytes([0, 8])                                        # Int64 (n_frag)
    out += bytes([16, 80]) + CORE + i32(2)                      # Array{F8, 2} (id 4)
    out += bytes([16]) + sym("Float8_E4M3FN")                   #   Float8_E4M3FN (id 5), name (id 6)
    out += bytes([31, 11]) + UUID.to_bytes(16, "little")        #   MODULE, UInt128 UUID
    out += sym("DLFP8Types") + bytes([68])                      #   :DLFP8Types (id 7), ()
    out += bytes([225])                                         #   N = 2 (Int64 literal)
    out += bytes([16, 80]) + CORE + i32(2) + bytes([0, 13, 225])  # Array{Float32, 2} (id 8)
    out += bytes([16, 80]) + CORE + i32(2) + bytes([0, 33, 224])  # Array{String, 1} (id 9)
    out += bytes([16, 80]) + CORE + i32(2) + bytes([0, 8, 224])   # Array{Int64, 1} (id 10)
    out += bytes([16, 80]) + CORE + i32(2) + bytes([0, 3, 224])   # Array{UInt8, 1} (id 11)
    # the 15 values
    out += bytes([57]) + string(FORMAT)                         # format: SHARED_REF (id 12), STRING
    out += bytes([57]) + string(SOURCE)                         # source (id 13)
    out += bytes([223 + K, 223 + KSTEP, 223 + S, 223 + M, 223 + C, 223 + 0])  # k kstep s m c normalize
    out += bytes([77])                                          # fp8 = true
    out += bytes([223 + N // 2])                                # n_frag
    out += bytes([21, 44]) + struct.pack("<H", 5)               # embeds8 (id 14): ARRAY, eltype = backref 5
    out += bytes([20, 2, 223 + RDIM, 223 + N]) + EMBEDS8        #   dims (8, 4), 32 bytes column-major
    out += bytes([21, 0, 13, 20, 2, 223 + M, 223 + N])          # norms (id 15): Float32, dims (1, 4)
    out += b"".join(struct.pack("<f", v) for v in NORMS)
    out += bytes([21, 0, 33, 223 + N])                          # heads (id 16): String, length 4
    out += bytes([57]) + string(HEADS[0])                       #   first ">chrA tiny" (id 17)
    out += bytes([44]) + struct.pack("<H", 17)                  #   again: SHORTBACKREF 17
    out += bytes([44]) + struct.pack("<H", 17)
    out += string(HEADS[3])                                     #   ">B" (<= 7 bytes: inline, no id)
    out += bytes([21, 0, 8, 223 + N])                           # starts (id 18): Int64, length 4
    out += b"".join(struct.pack("<q", v) for v in STARTS)
    out += bytes([21, 223 + N]) + bytes(STRAND)                 # strand (id 19): UInt8 (no eltype)
    return bytes(out)


if __name__ == "__main__":
    (HERE / "index_tiny.bin").write_bytes(build())
    print(f"wrote {HERE / 'index_tiny.bin'}")
