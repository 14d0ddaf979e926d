"""Build recipe for the CPU oracle (test infrastructure, see lssph_oracle.cpp).

    python oracle/build.py            -> oracle/_build/liblssph_oracle.so

Flags follow the reference's gfortran option (Makefile:51-54: -O2 -fopenmp) with
-ffp-contract=off so that only the explicit fma() calls of the restatement fuse, and
x86-64-v3 (AVX2+FMA) instead of -march=native so the library also runs on the host of
another machine.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "lssph_oracle.cpp")
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "liblssph_oracle.so")

FLAGS = ["-O2", "-march=x86-64-v3", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
         "-std=c++17", "-Wall", "-Wno-unused-function"]


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    hdr = os.path.join(HERE, "..", "include", "lssph.h")
    if not force and os.path.exists(OUT):
        newest = max(os.path.getmtime(SRC), os.path.getmtime(hdr))
        if os.path.getmtime(OUT) >= newest:
            return OUT
    cmd = ["g++", *FLAGS, SRC, "-o", OUT]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
