"""Builds the CPU oracle (test infrastructure only) into oracle/liboracle.so.

The oracle links the LAPACK/BLAS bundled with SciPy (libscipy_openblas, which
exports scipy_zgetrf_/scipy_zgetrs_/scipy_zgemm_), so it issues the same
zgetrf + zgetrs + zgemm sequence as the reference's CPU path.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def openblas_path():
    import scipy
    libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError("scipy's bundled OpenBLAS not found in %s" % libdir)
    return cands[0]


def build(force=False):
    src = os.path.join(HERE, "negf_oracle.cpp")
    hdr = os.path.join(os.path.dirname(HERE), "include", "negf_b200.h")
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(src), os.path.getmtime(hdr))):
        return LIB
    blas = openblas_path()
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", src, "-o", LIB,
           "-L" + os.path.dirname(blas), "-l:" + os.path.basename(blas),
           "-Wl,-rpath," + os.path.dirname(blas)]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
