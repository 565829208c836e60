"""Writes tests/golden/golden.npz: seeded small devices (their blocks stored
verbatim, so the fixture does not depend on the generators staying the same)
and the oracle's outputs on them.

The reference's own golden data (tests/f90Si*/transmission_ref.dat,
tests/f90elph_deph, f90sgf_cache) are git-lfs pointers without content, so
these fixtures pin the CPU restatement of the reference algorithm at one
point in time.  `tests/test_golden.py` checks that the oracle still
reproduces them (CPU) and that the CUDA path matches them (GPU).

Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libnegf_b200 import generators as G      # noqa: E402
from libnegf_b200.density import contour_points  # noqa: E402
from libnegf_b200.device import Device        # noqa: E402
from oracle import oracle as O                # noqa: E402

BLOCK_LISTS = ("h_diag", "h_upper", "h_lower", "s_diag", "s_upper", "s_lower",
               "lead_h00", "lead_h01", "lead_s00", "lead_s01", "hmc", "smc")


def store_device(out, name, dev):
    out[name + "__cblk"] = np.asarray(dev.cblk, dtype=np.int32)
    for k in BLOCK_LISTS:
        lst = getattr(dev, k)
        if lst is None:
            continue
        out["%s__%s__n" % (name, k)] = np.int32(len(lst))
        for i, b in enumerate(lst):
            out["%s__%s__%d" % (name, k, i)] = np.asarray(b, dtype=np.complex128)


def load_device(z, name):
    kw = {}
    for k in BLOCK_LISTS:
        key = "%s__%s__n" % (name, k)
        if key in z:
            kw[k] = [np.array(z["%s__%s__%d" % (name, k, i)]) for i in range(int(z[key]))]
        else:
            kw[k] = None
    return Device(kw["h_diag"], kw["h_upper"], kw["h_lower"], [int(c) for c in z[name + "__cblk"]],
                  kw["lead_h00"], kw["lead_h01"], kw["hmc"], s_diag=kw["s_diag"], s_upper=kw["s_upper"],
                  s_lower=kw["s_lower"], lead_s00=kw["lead_s00"], lead_s01=kw["lead_s01"], smc=kw["smc"])


def cases():
    """(name, device, dict of run parameters); the runs are in `run_case`."""
    return [
        ("c0_tdos", G.transport_c0(nbl=6, n=12, seed=21),
         dict(kind="tdos", E=np.linspace(-3.0, 3.0, 25), eta=1e-4, dos_delta=1e-4)),
        ("c0_t_eta6", G.transport_c0(nbl=6, n=12, seed=21),
         dict(kind="t", E=np.linspace(-2.9, 2.9, 21), eta=1e-6)),
        ("c1_tdos", G.transport_c1(nbl=5, n=16, seed=5, kpoint=0.3),
         dict(kind="tdos", E=np.linspace(-2.0, 2.0, 17), eta=1e-4, dos_delta=1e-4)),
        ("three_pairs", G.transport_c0(nbl=6, n=8, seed=1, cblk=[1, 6, 3]),
         dict(kind="pairs", E=np.linspace(-2.5, 2.5, 11), eta=1e-4, pairs=[(1, 2), (1, 3), (2, 3)],
              dos_proj=[[1, 2, 3], list(range(9, 17)), [40, 48]], dos_delta=1e-4)),
        ("scba", G.transport_c0(nbl=6, n=8, seed=4),
         dict(kind="scba", E=np.linspace(-1.0, 1.0, 9), eta=1e-4, frm=[1.0, 0.0], coupling=0.05, niter=5)),
        ("rho_eq", G.transport_c0(nbl=4, n=8, seed=9),
         dict(kind="rho", elow=-4.0, mu=0.0, kT=0.025, nkt=10, np1=8, np2=12, npoles=3)),
    ]


def run_case(dev, p):
    """The oracle outputs of one case, as a dict of arrays."""
    if p["kind"] == "tdos":
        T, dos, nc, st = O.transmission_dos(dev, p["E"], eta=p["eta"], dos_delta=p["dos_delta"])
        return dict(T=T, dos=dos, ncyc=nc, status=st)
    if p["kind"] == "t":
        T, nc, st = O.transmission(dev, p["E"], eta=p["eta"])
        return dict(T=T, ncyc=nc, status=st)
    if p["kind"] == "pairs":
        T, led, nc, st = O.transmissions(dev, p["E"], p["pairs"], eta=p["eta"], dos_proj=p["dos_proj"],
                                         dos_delta=p["dos_delta"])
        return dict(T=T, ledos=led, ncyc=nc, status=st)
    if p["kind"] == "scba":
        r = O.meir_wingreen(dev, p["E"], p["frm"], coupling=np.full(dev.norb, p["coupling"]), eta=p["eta"],
                            scba_niter=p["niter"])
        return dict(curr=r["curr"], layer_curr=r["layer_curr"], layer_dens=r["layer_dens"],
                    scba_iter=r["scba_iter"], ncyc=r["ncyc"], status=r["status"])
    if p["kind"] == "rho":
        z, w = contour_points(p["elow"], p["mu"], p["kT"], p["nkt"], p["np1"], p["np2"], p["npoles"])
        (d, u, l), _, nc, st = O.density(dev, z, w)
        return dict(z=np.asarray(z), w=np.asarray(w), rho_diag=np.stack(d), rho_upper=np.stack(u),
                    rho_lower=np.stack(l), ncyc=nc, status=st)
    raise ValueError(p["kind"])


def main():
    out = {}
    for name, dev, p in cases():
        store_device(out, name, dev)
        for k, v in run_case(dev, p).items():
            out["%s__out__%s" % (name, k)] = np.asarray(v)
    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **out)
    print("wrote %s (%d arrays, %d bytes)" % (path, len(out), os.path.getsize(path)))


if __name__ == "__main__":
    main()
