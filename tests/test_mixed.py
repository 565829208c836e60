"""The mixed-precision form (options.precision != 0): 2-contact transmission
with every block product on the integer tensor cores (int8 digits, exact int32
accumulation, FP64 recombination), block inverses, the decimation's
convergence test and the Caroli trace in FP64, all points of a call in lock
step.

Bound (the mixed form's target): |T - T_oracle| <= max(1e-8 |T_oracle|, 1e-11),
strict wherever the CPU FP64 paths of the same algorithm lie within an eighth
of it from the long-double solution; the decimation's iteration counts equal
the oracle's."""
import numpy as np
import pytest

from conftest import assert_parity, oracle_spread, xp_reference
from golden.make_config_shapes import CASES, PATH, fingerprint
from libnegf_b200 import generators as G
from libnegf_b200 import native
from oracle import oracle as O

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-8, 1e-11


def _bound(Tref):
    return np.maximum(RTOL * np.abs(Tref), ATOL)


def _mixed_T(ctx, hid, E, eta, digits=8, sgf_tol=1e-9):
    ctx.set_options(precision=digits, sgf_tol=sgf_tol)
    try:
        return ctx.transmission(hid, E, eta=eta, check=False)
    finally:
        ctx.set_options()


@pytest.mark.parametrize("gen", ["c0", "c1_S"])
def test_mixed_transmission_against_oracle(gpu_ctx, gen):
    dev = (G.transport_c0(nbl=6, n=128, seed=3) if gen == "c0"
           else G.transport_c1(nbl=5, n=128, seed=3, density=0.2))
    E = np.linspace(-2.5, 2.5, 24) if gen == "c0" else np.linspace(-1.8, 1.8, 24)
    did = gpu_ctx.upload(dev)
    try:
        T, ncyc, st = _mixed_T(gpu_ctx, did, E, 1e-6)
        ref, spread = oracle_spread(lambda d: dict(zip(("T", "ncyc", "status"), O.transmission(d, E, eta=1e-6))),
                                    dev, nsamp=2)
        assert np.all(st == ref["status"])
        assert np.array_equal(ncyc, ref["ncyc"])
        x = xp_reference(dev, E, 1e-6)
        assert_parity(T, ref["T"], _bound(ref["T"]), ref_x=x["T_x"], others=(x["T_d"], x["T_g"]),
                      spread=spread["T"], what="mixed T")
    finally:
        gpu_ctx.release(did)


def test_mixed_equals_plain_fp64_form_within_bound(gpu_ctx):
    """The mixed form against the plain FP64 GPU form, several k-points of one
    device in one call (points of different devices in a batch)."""
    devs = G.transport_c1_kpoints([0.0, 0.7, 1.9], nbl=4, n=128, seed=5, density=0.2)
    E = np.linspace(-1.5, 1.5, 10)
    hs = [gpu_ctx.upload(d) for d in devs]
    try:
        ids = np.repeat(np.asarray(hs, dtype=np.int32), E.size)
        EE = np.tile(E, len(hs))
        Tm, ncm, stm = _mixed_T(gpu_ctx, ids, EE, 1e-6)
        Tp, ncp, stp = gpu_ctx.transmission(ids, EE, eta=1e-6)
        assert np.all(stm == 0) and np.all(stp == 0)
        assert np.array_equal(ncm, ncp)
        for k, d in enumerate(devs):
            sl = slice(k * E.size, (k + 1) * E.size)
            ref, spread = oracle_spread(lambda dd: {"T": O.transmission(dd, E, eta=1e-6)[0]}, d, nsamp=2)
            x = xp_reference(d, E, 1e-6)
            assert_parity(Tm[sl], ref["T"], _bound(ref["T"]), ref_x=x["T_x"], others=(x["T_d"], x["T_g"]),
                          spread=spread["T"], what="mixed k=%d" % k)
    finally:
        for h in hs:
            gpu_ctx.release(h)


def test_mixed_at_the_c2_shape(gpu_ctx):
    """60 layers x 512 orbitals, S != I, eta = 1e-6: four grid energies over two
    k-points and four within 1e-3 eV of a lead band edge (fixture)."""
    z = np.load(PATH)
    devs, ids, E, p = CASES["c2"]()
    for k, d in enumerate(devs):
        assert fingerprint(d) == str(z["c2__fp%d" % k])
    E = np.array(z["c2__E"])   # band-edge energies: the fixture's (eigensolver bits differ across hosts)
    hs = [gpu_ctx.upload(d) for d in devs]
    try:
        hid = np.asarray(hs, dtype=np.int32)[ids]
        T, ncyc, st = _mixed_T(gpu_ctx, hid, E, p["eta"], sgf_tol=p["sgf_tol"])
        assert np.all(st == 0)
        assert np.array_equal(ncyc, z["c2__ncyc_o"])
        Tr = z["c2__T_o"]
        listed = assert_parity(T, Tr, _bound(Tr), ref_x=z["c2__T_x"], others=(z["c2__T_d"], z["c2__T_g"]),
                               spread=z["c2__T_s"], what="mixed c2")
        print("mixed c2: max rel err %.2e, %d listed" % ((np.abs(T - Tr) / np.abs(Tr)).max(), listed.size))
    finally:
        for h in hs:
            gpu_ctx.release(h)


def test_mixed_rejects_what_it_does_not_cover(gpu_ctx):
    dev = G.transport_c0(nbl=6, n=8, seed=1, cblk=[2, 5])    # contacts off blocks 1 and nbl
    uneven = G.uneven([5, 7, 3, 6], seed=4)
    E = np.linspace(-1, 1, 3)
    d1, d2 = gpu_ctx.upload(dev), gpu_ctx.upload(uneven)
    ok = gpu_ctx.upload(G.transport_c0(nbl=3, n=16, seed=2))
    gpu_ctx.set_options(precision=8)
    try:
        for did in (d1, d2):
            with pytest.raises(native.NegfError) as e:
                gpu_ctx.transmission(did, E, eta=1e-6)
            assert e.value.code == native.BAD_ARG
        with pytest.raises(native.NegfError) as e:   # DOS is the FP64 engine's
            gpu_ctx.transmission_dos(ok, E, eta=1e-6)
        assert e.value.code == native.BAD_ARG
    finally:
        gpu_ctx.set_options()
        for h in (d1, d2, ok):
            gpu_ctx.release(h)
