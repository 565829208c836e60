"""Edge cases of the per-point solve: empty calls, a single contact, ragged
layer sizes across the register-leaf shapes (1, 2 and 4 rows per thread),
and the decimation iteration cap."""
import numpy as np
import pytest

from conftest import assert_T_close, oracle_spread
from libnegf_b200 import generators as G
from oracle import oracle as O


def test_single_contact_oracle_gives_zero():
    dev = G.transport_c0(nbl=3, n=4, seed=3, cblk=[1])
    T, _, st = O.transmission(dev, np.linspace(-1, 1, 5), eta=1e-4, ni=1, nf=1)
    assert np.all(T == 0.0) and np.all(st == 0)


@pytest.mark.gpu
def test_empty_call(gpu_ctx):
    dev = G.transport_c0(nbl=3, n=4, seed=3)
    did = gpu_ctx.upload(dev)
    try:
        T, nc, st = gpu_ctx.transmission(did, np.zeros(0), eta=1e-4)
        assert T.size == 0 and nc.size == 0 and st.size == 0
        T, led, nc, st = gpu_ctx.transmissions(did, np.zeros(0), [(1, 2), (2, 1)], eta=1e-4)
        assert T.shape == (0, 2)
    finally:
        gpu_ctx.release(did)


@pytest.mark.gpu
def test_single_contact(gpu_ctx):
    """ncont = 1: T = 0 (src/iterative.F90:1684-1687); the DOS is still solved."""
    dev = G.transport_c0(nbl=3, n=4, seed=3, cblk=[1])
    E = np.linspace(-2, 2, 9)
    did = gpu_ctx.upload(dev)
    try:
        T, nc, st = gpu_ctx.transmission(did, E, eta=1e-4, ni=1, nf=1)
        assert np.all(T == 0.0) and np.all(st == 0)
        Td, dos, _, st = gpu_ctx.transmission_dos(did, E, eta=1e-4, dos_delta=1e-4, ni=1, nf=1)
        ref = O.transmission_dos(dev, E, eta=1e-4, dos_delta=1e-4, ni=1, nf=1)
        assert np.all(Td == 0.0)
        assert np.abs(dos - ref[1]).max() <= 1e-10 * max(1.0, np.abs(ref[1]).max())
    finally:
        gpu_ctx.release(did)


@pytest.mark.gpu
def test_ragged_layers_across_leaf_shapes(gpu_ctx):
    """PL sizes 300 (2 rows per thread in the leaves), 40 (whole matrix in
    shared memory) and 520 (4 rows per thread) in one device."""
    dev = G.uneven([300, 40, 520], seed=8)
    E = np.array([-0.7, 0.3])
    did = gpu_ctx.upload(dev)
    try:
        T, nc, st = gpu_ctx.transmission(did, E, eta=1e-4)
        # ill-conditioned: 1e-15 input perturbations move the oracle's T by up to ~1e-8 here,
        # so the spread needs a few samples to be representative
        ref, spread = oracle_spread(lambda d: O.transmission(d, E, eta=1e-4)[0], dev, nsamp=4)
        assert np.all(st == O.transmission(dev, E, eta=1e-4)[2])
        assert_T_close(T, ref, spread=spread)
    finally:
        gpu_ctx.release(did)


@pytest.mark.gpu
def test_decimation_iteration_cap(gpu_ctx):
    """A cap too small to converge: NOT_CONVERGED on the same points as the
    oracle, with the same (unconverged) result."""
    dev = G.transport_c0(nbl=4, n=8, seed=0)
    E = np.linspace(-2.5, 2.5, 9)
    did = gpu_ctx.upload(dev)
    try:
        gpu_ctx.set_options(sgf_max_iter=3)
        T, nc, st = gpu_ctx.transmission(did, E, eta=1e-4, check=False)
        ref, spread = oracle_spread(lambda d: O.transmission(d, E, eta=1e-4, sgf_max_iter=3)[0], dev)
        rst = O.transmission(dev, E, eta=1e-4, sgf_max_iter=3)[2]
        assert np.array_equal(st, rst) and np.any(st == 2)
        assert_T_close(T, ref, spread=spread)
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)


@pytest.mark.gpu
@pytest.mark.parametrize("where", ["device", "lead"])
def test_nonfinite_input_gives_a_status_not_a_trap(gpu_ctx, where):
    """A NaN planted on the host in H (a device block, or a lead block) comes
    back as a non-finite result with a non-zero per-point status for every
    point, through the FP64 engine and the mixed form alike; the context
    stays usable: a clean device solved right after matches the oracle.  The
    reference has no such status (its GPU path sums |A| to look for NaN and
    stops, src/gpuroutines.cu:697-739)."""
    bad = G.transport_c0(nbl=4, n=128, seed=8)
    if where == "device":
        bad.h_diag[2][5, 7] = np.nan
    else:
        bad.lead_h00[0][3, 3] = np.nan
    E = np.linspace(-1.5, 1.5, 6)
    clean = G.transport_c0(nbl=4, n=128, seed=9)
    b, c = gpu_ctx.upload(bad), gpu_ctx.upload(clean)
    try:
        for precision in (0, 8):
            gpu_ctx.set_options(precision=precision)
            T, nc, st = gpu_ctx.transmission(b, E, eta=1e-6, check=False)
            assert np.all(st != 0), (precision, st)
            assert not np.isfinite(T).all() or np.all(st == 3), (precision, T, st)
            T2, nc2, st2 = gpu_ctx.transmission(c, E, eta=1e-6)
            assert np.all(st2 == 0)
            Tr, ncr, _ = O.transmission(clean, E, eta=1e-6)
            assert np.array_equal(nc2, ncr)
            assert np.all(np.abs(T2 - Tr) <= np.maximum(1e-8 * np.abs(Tr), 1e-11))
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(b)
        gpu_ctx.release(c)
