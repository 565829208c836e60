"""Builds the CUDA extension libnegf_b200.so in-tree for sm_100a.

Plain nvcc, no JIT cache: the shared object is written next to this file so
that it travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libnegf_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("engine.cu", "program.cu", "capi.cu", "noalloc.cu", "gemm_dev.cu", "leaf_dev.cu",
                                                     "csr.cu", "ozaki.cu", "mixed.cu", "small.cu")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in ("cta_ops.cuh", "engine.cuh", "program.cuh", "ozaki.cuh", "mixed.cuh", "small.cuh")] + [
    os.path.join(ROOT, "include", "negf_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def build(force=False, verbose=False):
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(p) for p in DEPS)):
        return LIB
    # relocatable device code: the engine kernel with its inlined product
    # loop, the control code (program.cu) and the inversion leaves
    # (leaf_dev.cu) are register-allocated apart from one another
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-rdc=true", "-Xptxas=--device-function-maxrregcount=128",
           "-shared", "-Xcompiler", "-fPIC",
           "-I" + os.path.join(ROOT, "include"), *SOURCES, "-o", LIB]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
