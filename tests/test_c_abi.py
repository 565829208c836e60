"""The C-ABI driven from C: tests/c_abi/negf_c_check.c, built here with gcc
against include/negf_b200.h and libnegf_b200.so, fills a negf_b200_device
itself and calls negf_b200_transmission; its T must match the oracle (the
strict parity rule of the Python-driven tests) and its decimation counts
the oracle's.  This pins the struct layout and the by-value / by-pointer
arguments as a C (or Fortran bind(C)) caller sees them."""
import os
import subprocess

import numpy as np
import pytest

from conftest import assert_T_strict, oracle_spread, xp_reference
from libnegf_b200 import generators as G
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "c_abi", "negf_c_check.c")
LIBDIR = os.path.join(ROOT, "libnegf_b200")


def _write_device(path, dev):
    has_s = dev.s_diag is not None
    with open(path, "wb") as f:
        np.asarray([dev.nbl, dev.ncont, int(has_s)], dtype=np.int32).tofile(f)
        np.asarray([b.shape[0] for b in dev.h_diag], dtype=np.int32).tofile(f)
        np.asarray(dev.cblk, dtype=np.int32).tofile(f)
        np.asarray([b.shape[0] for b in dev.lead_h00], dtype=np.int32).tofile(f)
        fam = [dev.h_diag, dev.h_upper, dev.h_lower]
        if has_s:
            fam += [dev.s_diag, dev.s_upper, dev.s_lower]
        fam += [dev.lead_h00, dev.lead_h01]
        if has_s:
            fam += [dev.lead_s00, dev.lead_s01]
        fam += [dev.hmc]
        if has_s:
            fam += [dev.smc]
        for lst in fam:
            for b in lst:
                np.ascontiguousarray(np.asarray(b, dtype=np.complex128).ravel(order="F")).view(np.float64).tofile(f)


def build_c_check(tmp):
    exe = os.path.join(tmp, "negf_c_check")
    subprocess.check_call(["gcc", "-O2", "-std=c11", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), SRC,
                           "-L" + LIBDIR, "-lnegf_b200", "-Wl,-rpath," + LIBDIR, "-o", exe])
    return exe


def test_c_program_compiles_against_the_header(tmp_path):
    """CPU: the header is valid C11 and the program links against the library."""
    if not os.path.exists(os.path.join(LIBDIR, "libnegf_b200.so")):
        pytest.skip("libnegf_b200.so not built")
    assert os.path.exists(build_c_check(str(tmp_path)))


@pytest.mark.gpu
@pytest.mark.parametrize("gen", ["c0", "c1_S"])
def test_c_program_transmission_matches_oracle(tmp_path, gen):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    dev = (G.transport_c0(nbl=6, n=16, seed=12) if gen == "c0"
           else G.transport_c1(nbl=5, n=12, seed=2, density=0.3))
    E = np.linspace(-2.0, 2.0, 17)
    eta = 1e-6
    exe = build_c_check(str(tmp_path))
    dpath, epath, opath = (str(tmp_path / n) for n in ("dev.bin", "E.bin", "out.bin"))
    _write_device(dpath, dev)
    with open(epath, "wb") as f:
        np.asarray([E.size], dtype=np.int32).tofile(f)
        np.asarray([eta], dtype=np.float64).tofile(f)
        E.astype(np.float64).tofile(f)
    r = subprocess.run([exe, dpath, epath, opath], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = open(opath, "rb").read()
    T = np.frombuffer(raw[:8 * E.size], dtype=np.float64)
    ncyc = np.frombuffer(raw[8 * E.size:12 * E.size], dtype=np.int32)
    st = np.frombuffer(raw[12 * E.size:], dtype=np.int32)
    ref, spread = oracle_spread(lambda d: dict(zip(("T", "ncyc", "status"), O.transmission(d, E, eta=eta))), dev,
                                nsamp=2)
    assert np.array_equal(st, ref["status"])
    assert np.array_equal(ncyc, ref["ncyc"])
    assert_T_strict(T, ref["T"], xp_reference(dev, E, eta), spread=spread["T"], what="C caller")
