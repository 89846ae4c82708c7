"""Builds the engine's shared library (libmxg.so) for sm_100a with nvcc.

The library holds the CUDA kernels, the host engine and the table builder,
and exports the C ABI declared in include/mxg.h. It is built in-tree so it
ships with the package directory.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmxg.so")

SOURCES = ["mxg_kernels.cu", "mxg_adjoint.cu", "mxg_pairs.cu", "mxg_metrics.cu", "mxg_engine.cpp", "potential_table.cpp",
           "mxg_noalloc.cu"]
HEADERS = ["mxg_device.cuh", "mxg_kernels.h", "potential_table.h", "mxg_adjoint.h"]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "mxg.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    cmd = [
        nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
        # every device FP op rounds separately, as the reference's scalar CPU code does
        "-fmad=false",
        "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
        "-shared", "-o", LIB,
    ] + [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=HERE)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
