"""Build recipe of the engine library (sm_100a).

    python ls-sph-benchmarks_b200/build.py      -> ls-sph-benchmarks_b200/lib/liblssph.so

nvcc cross-compiles here without a GPU.  The device code is compiled with -fmad=false:
the FP64 kernels place every fused multiply-add explicitly (fma()), in the same places
as the CPU restatement they are checked against.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "liblssph.so")
INCLUDE = os.path.join(HERE, "..", "include")

SOURCES = ["host.cpp", "engine.cu", "split_shape.cu", "batch.cu", "noalloc.cu", "highorder.cu", "postproc.cu",
           "snapshot.cu"]
HEADERS = ["engine.h", "handle.h", "hostmem.h", "kernels.cuh", "kernels_hi.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-O2,-Wall",
]
OBJ_DIR = os.path.join(LIB_DIR, "_obj")


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(INCLUDE, "lssph.h"), os.path.abspath(__file__)]
    newest = max(os.path.getmtime(d) for d in deps if os.path.exists(d))
    return os.path.getmtime(LIB) < newest


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    """Compile each source to an object in parallel, then link the shared library."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(OBJ_DIR, exist_ok=True)
    base = [_nvcc(), *NVCC_FLAGS] + (["-Xptxas", "-v"] if verbose_ptxas else []) + ["-I", INCLUDE]

    def compile_one(src: str) -> str:
        obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        subprocess.run([*base, "-c", os.path.join(CSRC, src), "-o", obj], check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    subprocess.run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs,
                    "-o", LIB + ".tmp"], check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
