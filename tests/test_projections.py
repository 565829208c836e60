"""Contact pairs, tun_proj and dos_proj: the oracle's own consistency (CPU)
and the GPU engine against the oracle (gpu).

Reference behaviour (libNEGF): calculate_transmissions loops over the pairs
ni(:), nf(:) (src/iterative.F90:1669-1780), both transmission formulas trace
over the tun_proj mask of get_tun_mask (src/iterative_cpu.F90:586-618) and
calculate_transmissions_and_dos sums -Im Gr_ii / pi over every dos_proj set
(src/iterative.F90:1931-1945)."""
import numpy as np
import pytest

from conftest import assert_T_close, oracle_spread
from libnegf_b200 import generators as G
from libnegf_b200.projections import dos_sets, tun_mask
from oracle import oracle as O


def three_contacts():
    # contacts on blocks 1, 6 and 3 of a 6-layer device
    return G.transport_c0(nbl=6, n=8, seed=1, cblk=[1, 6, 3]), np.linspace(-2.5, 2.5, 11)


PAIRS3 = [(1, 2), (1, 3), (3, 2), (2, 1)]
TUN3 = list(range(1, 5)) + list(range(17, 21)) + list(range(41, 45))
SETS3 = [[1, 2, 3], list(range(9, 17)), [48, 47, 100], list(range(1, 49))]


def test_projection_helpers():
    m = tun_mask(6, [1, 3, 3, 9, 0])
    assert m.tolist() == [1, 0, 1, 0, 0, 0]
    assert tun_mask(4, None) is None
    ptr, idx = dos_sets([[2, 1], [], [5]])
    assert ptr.tolist() == [0, 2, 2, 3] and idx.tolist() == [2, 1, 5]


def test_oracle_pairs_equal_single_pair_calls():
    dev, E = three_contacts()
    T, _, _, st = O.transmissions(dev, E, PAIRS3, eta=1e-6)
    assert np.all(st == 0)
    for q, (a, b) in enumerate(PAIRS3):
        t1, _, _ = O.transmission(dev, E, eta=1e-6, ni=a, nf=b)
        assert np.array_equal(t1, T[:, q])
    # reciprocity of the N-contact formula for a pair and its reverse
    assert np.allclose(T[:, 0], T[:, 3], rtol=0, atol=1e-12)


def test_oracle_full_tun_proj_equals_no_projection():
    dev, E = three_contacts()
    T0, _, _, _ = O.transmissions(dev, E, PAIRS3, eta=1e-6)
    T1, _, _, _ = O.transmissions(dev, E, PAIRS3, eta=1e-6, tun_proj=range(1, dev.norb + 1))
    assert np.array_equal(T0, T1)
    d2 = G.transport_c0(nbl=5, n=6, seed=2)
    E2 = np.linspace(-2, 2, 7)
    t0, _, _ = O.transmission(d2, E2, eta=1e-6)
    t1, _, _, _ = O.transmissions(d2, E2, [(1, 2)], eta=1e-6, tun_proj=range(1, d2.norb + 1))
    assert np.array_equal(t0, t1[:, 0])


def test_oracle_ldos_sets_are_sums_of_the_dos():
    dev, E = three_contacts()
    T, dos, _, _ = O.transmission_dos(dev, E, eta=1e-6, dos_delta=1e-4, ni=1, nf=2)
    T2, led, _, _ = O.transmissions(dev, E, [(1, 2)], eta=1e-6, dos_proj=SETS3, dos_delta=1e-4)
    assert np.array_equal(T, T2[:, 0])
    for k, s in enumerate(SETS3):
        ok = [i - 1 for i in s if 1 <= i <= dev.norb]
        assert np.allclose(led[:, k], dos[:, ok].sum(axis=1), rtol=1e-13, atol=1e-15)


# ------------------------------------------------------------------ GPU parity
def _o_pairs(E, pairs, **kw):
    def run(d):
        T, led, nc, st = O.transmissions(d, E, pairs, **kw)
        out = {"T": T, "ncyc": nc, "status": st}
        if led is not None:
            out["ldos"] = led
        return out
    return run


@pytest.mark.gpu
@pytest.mark.parametrize("tun", [None, TUN3])
def test_pairs_parity(gpu_ctx, tun):
    dev, E = three_contacts()
    did = gpu_ctx.upload(dev)
    try:
        gpu_ctx.set_tun_proj(did, tun)
        T, _, ncyc, st = gpu_ctx.transmissions(did, E, PAIRS3, eta=1e-6)
        ref, spread = oracle_spread(_o_pairs(E, PAIRS3, eta=1e-6, tun_proj=tun), dev)
        assert np.all(st == ref["status"])
        assert_T_close(T, ref["T"], spread=spread["T"])
    finally:
        gpu_ctx.release(did)


@pytest.mark.gpu
@pytest.mark.parametrize("tun", [None, TUN3])
def test_pairs_ldos_parity(gpu_ctx, tun):
    dev, E = three_contacts()
    did = gpu_ctx.upload(dev)
    try:
        gpu_ctx.set_tun_proj(did, tun)
        gpu_ctx.set_dos_proj(did, SETS3)
        T, led, ncyc, st = gpu_ctx.transmissions(did, E, PAIRS3, eta=1e-6, ldos=True, dos_delta=1e-4)
        ref, spread = oracle_spread(_o_pairs(E, PAIRS3, eta=1e-6, tun_proj=tun, dos_proj=SETS3, dos_delta=1e-4), dev)
        assert np.all(st == ref["status"])
        assert_T_close(T, ref["T"], spread=spread["T"])
        scale = max(np.abs(ref["ldos"]).max(), 1.0)
        assert np.all(np.abs(led - ref["ldos"]) <= np.maximum(1e-10 * scale, 10 * spread["ldos"]))
    finally:
        gpu_ctx.release(did)


@pytest.mark.gpu
@pytest.mark.parametrize("ldos", [False, True])
def test_tun_proj_two_contacts(gpu_ctx, ldos):
    """The 2-contact formula (fast path in the T solve) with a projection."""
    dev = G.transport_c0(nbl=6, n=8, seed=0)
    E = np.linspace(-3, 3, 13)
    tun = list(range(1, 5))
    sets = [[1, 2], list(range(1, dev.norb + 1))]
    did = gpu_ctx.upload(dev)
    try:
        gpu_ctx.set_tun_proj(did, tun)
        gpu_ctx.set_dos_proj(did, sets)
        T, led, _, st = gpu_ctx.transmissions(did, E, [(2, 1)], eta=1e-6, ldos=ldos, dos_delta=1e-4)
        kw = dict(eta=1e-6, tun_proj=tun)
        if ldos:
            kw.update(dos_proj=sets, dos_delta=1e-4)
        ref, spread = oracle_spread(_o_pairs(E, [(2, 1)], **kw), dev)
        assert np.all(st == ref["status"])
        assert_T_close(T, ref["T"], spread=spread["T"])
        if ldos:
            scale = max(np.abs(ref["ldos"]).max(), 1.0)
            assert np.all(np.abs(led - ref["ldos"]) <= np.maximum(1e-10 * scale, 10 * spread["ldos"]))
        # clearing the projection restores the whole trace
        gpu_ctx.set_tun_proj(did, None)
        T0, _, _, _ = gpu_ctx.transmissions(did, E, [(2, 1)], eta=1e-6)
        Tf, _, _ = gpu_ctx.transmission(did, E, eta=1e-6, ni=2, nf=1)
        assert np.array_equal(T0[:, 0], Tf)
    finally:
        gpu_ctx.release(did)
