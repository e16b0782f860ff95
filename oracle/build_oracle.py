"""Build recipe for the CPU oracle (oracle/_build/libfire_oracle.so) -- test infrastructure only.

gcc, OpenMP, -O3, no FMA contraction (-ffp-contract=off) and no fast-math, so
the float instantiation rounds every operation exactly as written in the
reference's source.  The target is x86-64-v3 (AVX2/FMA-capable hosts) so the
library built here also runs on the GPU box's host.

Usage: python oracle/build_oracle.py
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build"
LIB = OUT / "libfire_oracle.so"
SOURCES = [HERE / "fire_oracle.cpp", HERE / "config_oracle.cpp"]
HEADERS = [HERE / "fire_oracle.h", HERE / "config_oracle.h", HERE.parent / "include" / "fire_cuda.h",
           HERE.parent / "include" / "fire_ext.h"]


def build(verbose: bool = False) -> Path:
    OUT.mkdir(parents=True, exist_ok=True)
    deps = SOURCES + HEADERS
    if LIB.exists() and all(LIB.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return LIB
    # The system g++ carries OpenMP; a CXX wrapper elsewhere on PATH may not.
    cxx = os.environ.get("FIRE_ORACLE_CXX", "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++")
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [cxx, "-std=c++17", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
           "-fPIC", "-shared", "-Wall", "-Wno-unused-function", *map(str, SOURCES), "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
    sys.exit(0)
