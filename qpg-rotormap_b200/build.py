"""Build librotormap_b200.so (sm_100a) in-tree with nvcc.

Usage: python qpg-rotormap_b200/build.py [--force] [--verbose]

The library lands in qpg-rotormap_b200/lib/librotormap_b200.so; object files
in qpg-rotormap_b200/_build/.  Sources are recompiled only when they (or a
header) changed.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "librotormap_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
           "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-I", str(CSRC)]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-I", str(ROOT / "include"), "-I", str(CSRC),
            "-I", "/usr/local/cuda/include"]


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers():
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted((ROOT / "include").glob("*.h"))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    hdr_mtime = max((p.stat().st_mtime for p in _headers()), default=0.0)
    objs = []
    for src in _sources():
        obj = OBJ / (src.name + ".o")
        objs.append(obj)
        if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_mtime):
            continue
        if src.suffix == ".cu":
            cmd = [NVCC, *ARCH, *CUFLAGS, "-c", str(src), "-o", str(obj)]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
        else:
            cmd = ["g++", *CXXFLAGS, "-c", str(src), "-o", str(obj)]
        _run(cmd, verbose)
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB), *map(str, objs),
               "-lpthread"]
        _run(cmd, verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv,
          ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
