"""Equilibrium density matrix by contour integration (contour_int_def +
contour_int): the host contour, the oracle's known answer, the blk2csr
restriction, and the device sum against the oracle (gpu)."""
import numpy as np
import pytest

from libnegf_b200 import density as D
from libnegf_b200 import generators as G
from libnegf_b200 import structure as St
from oracle import oracle as O

CONTOUR = dict(elow=-4.0, muref=0.0, kT=0.01, n_kt=10, np1=24, np2=12, n_poles=3)


def test_gauleg_matches_reference_convention():
    x, w = D.gauleg(np.pi, 0.3, 7)
    assert x[0] > x[-1] and np.all(np.diff(x) < 0)       # from x1 towards x2
    assert np.all(w < 0) and abs(w.sum() - (0.3 - np.pi)) < 1e-14
    # exact for polynomials of degree 2n-1
    x, w = D.gauleg(-1.0, 2.0, 4)
    assert abs(np.sum(w * x ** 7) - (2.0 ** 8 - 1.0) / 8.0) < 1e-12


def test_contour_layout():
    z, w = D.contour_points(**CONTOUR)
    assert z.size == 24 + 12 + 3
    assert np.all(z.imag > 0)                              # upper half plane
    poles = z[-3:]
    assert np.allclose(poles.imag, 0.01 * np.pi * np.array([1, 3, 5]))
    z0, _ = D.contour_points(elow=-4.0, muref=0.0, kT=0.0, n_kt=10, np1=8, np2=8, n_poles=0)
    assert z0.size == 16


def test_oracle_half_filled_chain_has_one_electron_per_site():
    """Perfect chain at mu = 0 (band centre): occupation g_spin / 2 = 1 per
    site by particle-hole symmetry."""
    dev = G.chain(1, 6)
    z, w = D.contour_points(**CONTOUR)
    (rd, ru, rl), (odc, ocd), nc, st = O.density(dev, z, w)
    assert np.all(st == 0)
    occ = np.array([b[0, 0].real for b in rd])
    assert np.allclose(occ, 1.0, atol=1e-10)
    for b in rd:
        assert np.abs(b - b.conj().T).max() < 1e-14
    for u, l in zip(ru, rl):
        assert np.abs(u - l.conj().T).max() < 1e-14


def test_oracle_chain_bond_order_inside_and_across_the_contacts():
    """Known answer for the equilibrium outer blocks (calculate_Gr_outer): in
    a half-filled perfect chain every nearest-neighbour density-matrix
    element is the bond order g_spin sin(k_F) / pi = 2 / pi, between device
    sites (upper blocks) and between the device's end sites and the first
    contact sites (outer blocks) alike; kT = 1e-3 moves it by O((pi kT)^2)."""
    dev = G.chain(1, 6)
    z, w = D.contour_points(elow=-4.0, muref=0.0, kT=0.001, n_kt=10, np1=48, np2=24, n_poles=3)
    (rd, ru, rl), (odc, ocd), nc, st = O.density(dev, z, w)
    assert np.all(st == 0)
    bonds = [b[0, 0] for b in ru] + [b[0, 0] for b in odc] + [b[0, 0] for b in ocd]
    assert np.allclose(bonds, 2.0 / np.pi, atol=1e-6)


def test_restrict_to_pattern_is_blk2csr():
    dev = G.transport_c1(nbl=3, n=5, seed=4, density=0.4)
    H, S, plend, *_ = St.csr_from_device(dev)
    d = [np.arange(25, dtype=complex).reshape(5, 5) + 100 * i for i in range(3)]
    u = [np.full((5, 5), 1000.0 + i, dtype=complex) for i in range(2)]
    l = [np.full((5, 5), 2000.0 + i, dtype=complex) for i in range(2)]
    R = D.restrict_to_pattern((d, u, l), S, plend).toarray()
    Sp = (S[:15, :15].toarray() != 0)
    full = np.zeros((15, 15), dtype=complex)
    for i in range(3):
        full[5 * i:5 * i + 5, 5 * i:5 * i + 5] = d[i]
    for i in range(2):
        full[5 * i:5 * i + 5, 5 * i + 5:5 * i + 10] = u[i]
        full[5 * i + 5:5 * i + 10, 5 * i:5 * i + 5] = l[i]
    assert np.array_equal(R, np.where(Sp, full, 0))


def _close(a, b, rel=1e-10):
    scale = max(max(np.abs(x).max() for x in b), 1.0)
    return all(np.abs(x - y).max() <= rel * scale for x, y in zip(a, b))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["chain", "c0", "uneven", "c1_S", "three"])
def test_density_parity(gpu_ctx, case):
    dev = {"chain": lambda: G.chain(1, 6),
           "c0": lambda: G.transport_c0(nbl=5, n=8, seed=1),
           "uneven": lambda: G.uneven([5, 9, 4, 7], seed=4),
           "c1_S": lambda: G.transport_c1(nbl=4, n=12, seed=2, density=0.3),
           "three": lambda: G.transport_c0(nbl=5, n=8, seed=1, cblk=[1, 5, 3])}[case]()
    z, w = D.contour_points(**CONTOUR)
    did = gpu_ctx.upload(dev)
    try:
        (gd, gu, gl), (gdc, gcd), nc, st = gpu_ctx.density(did, z, w)
        (od, ou, ol), (odc, ocd), onc, ost = O.density(dev, z, w)
        assert np.all(st == ost)
        assert _close(gd, od) and _close(gu, ou) and _close(gl, ol)
        assert _close(gdc, odc) and _close(gcd, ocd)
        for a, b in zip(odc, ocd):                               # rho is Hermitian across the outer blocks
            assert np.abs(a - b.conj().T).max() <= 1e-12 * max(1.0, np.abs(a).max())
        if case == "chain":
            assert np.allclose([b[0, 0].real for b in gd], 1.0, atol=1e-10)
    finally:
        gpu_ctx.release(did)


def test_oracle_real_axis_vanishes_in_equilibrium():
    dev = G.transport_c0(nbl=4, n=6, seed=1)
    E, w = D.real_axis_points(mu=[0.0, 0.0], kT=[0.01, 0.01], n_kt=10, np_real=12, delta=1e-4)
    frm = D.neq_occupations(E, [0.0, 0.0], [0.01, 0.01], ref=1)
    assert np.all(frm == 0.0)
    (rd, ru, rl), (rdc, rcd), nc, st = O.density_neq(dev, E, w, frm, eta=1e-4)
    assert all(np.abs(b).max() == 0.0 for b in rd + ru + rl + rdc + rcd)


@pytest.mark.gpu
@pytest.mark.parametrize("deph,three", [(False, False), (True, False), (False, True)])
def test_density_neq_parity(gpu_ctx, deph, three):
    """Tridiagonal blocks and the outer blocks of calculate_Gn_outer."""
    dev = G.transport_c0(nbl=4, n=6, seed=2, cblk=[1, 4, 2] if three else None)
    mu, kT = [0.1, -0.1], [0.01, 0.01]
    E, w = D.real_axis_points(mu=mu, kT=kT, n_kt=10, np_real=24, delta=1e-4)
    if three:
        mu, kT = mu + [0.05], kT + [0.01]
        E, w = D.real_axis_points(mu=mu, kT=kT, n_kt=10, np_real=24, delta=1e-4)
    frm = D.neq_occupations(E, mu, kT, ref=2)
    cpl = np.full(dev.norb, 0.05) if deph else None
    did = gpu_ctx.upload(dev)
    try:
        gpu_ctx.set_options(scba_niter=5 if deph else 0)
        (gd, gu, gl), (gdc, gcd), nc, st = gpu_ctx.density_neq(did, E, w, frm, eta=1e-4, coupling=cpl)
        (od, ou, ol), (odc, ocd), onc, ost = O.density_neq(dev, E, w, frm, eta=1e-4, coupling=cpl,
                                                           scba_niter=5 if deph else 0)
        assert np.all(st == ost)
        assert _close(gd, od, 1e-9) and _close(gu, ou, 1e-9) and _close(gl, ol, 1e-9)
        assert _close(gdc, odc, 1e-9) and _close(gcd, ocd, 1e-9)
        assert max(np.abs(b).max() for b in od) > 1e-4          # a bias window: a non-zero density
        assert max(np.abs(b).max() for b in odc) > 1e-6          # and non-zero outer blocks
        for a, b in zip(odc, ocd):                               # Gn(c,cb) = Gn(cb,c)^dag (real weights)
            assert np.abs(a - b.conj().T).max() <= 1e-12 * max(1.0, np.abs(a).max())
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)


def _bond_currents(dev, E, outer):
    """Current from device block cblk into each contact, from the outer
    blocks of one real-axis point: Re[i Tr(Tlc Gn(c,cb) - Gn(cb,c) Tcl)],
    Tlc = E SMC - HMC, Tcl = Tlc^dag (the layer-current formula of
    iterative_layer_current, src/iterative.F90:427-461, on the device-contact
    bond)."""
    dc, cd = outer
    J = []
    for c in range(dev.ncont):
        smc = dev.smc[c] if dev.smc is not None else 0.0
        Tlc = E * smc - dev.hmc[c]
        J.append(np.real(1j * np.trace(Tlc @ cd[c] - dc[c] @ Tlc.conj().T)))
    return np.array(J)


@pytest.mark.parametrize("case", ["two", "three", "c1_S"])
def test_oracle_outer_blocks_carry_the_contact_currents(case):
    """Known answer for calculate_Gn_outer: at one coherent real-axis point
    (weight 1) the bond current between device block cblk and each contact,
    formed from the outer blocks, is that contact's Meir-Wingreen current
    (exact with S = I; with an overlap the broadening eta on the contact
    side leaves an O(eta |S|) difference)."""
    dev = {"two": lambda: G.transport_c0(nbl=4, n=6, seed=2),
           "three": lambda: G.transport_c0(nbl=5, n=6, seed=1, cblk=[1, 5, 3]),
           "c1_S": lambda: G.transport_c1(nbl=4, n=8, seed=3, density=0.4)}[case]()
    nc = dev.ncont
    for E in (0.05, -0.3, 0.7):
        frm = np.array([[1.0] + [0.0] * (nc - 2) + [0.3]]) if nc > 2 else np.array([[1.0, 0.0]])
        _, outer, _, st = O.density_neq(dev, [E], np.array([1.0 + 0j]), frm, eta=1e-6, scba_niter=0)
        mw = O.meir_wingreen(dev, [E], frm, eta=1e-6, scba_niter=0)
        J = _bond_currents(dev, E, outer)
        tol = 1e-10 if case != "c1_S" else 1e-5
        assert np.abs(J - mw["curr"][0]).max() <= tol * max(1.0, np.abs(mw["curr"][0]).max())
        assert abs(J.sum()) <= tol                                  # current conservation


@pytest.mark.gpu
@pytest.mark.parametrize("three", [False, True])
def test_gpu_outer_blocks_carry_the_contact_currents(gpu_ctx, three):
    """The same known answer on the CUDA path's outer blocks."""
    dev = G.transport_c0(nbl=5, n=6, seed=1, cblk=[1, 5, 3]) if three else G.transport_c0(nbl=4, n=6, seed=2)
    nc = dev.ncont
    frm = np.array([[1.0] + [0.0] * (nc - 2) + [0.3]]) if nc > 2 else np.array([[1.0, 0.0]])
    did = gpu_ctx.upload(dev)
    try:
        gpu_ctx.set_options(scba_niter=0)
        for E in (0.05, -0.3, 0.7):
            _, outer, _, st = gpu_ctx.density_neq(did, [E], np.array([1.0 + 0j]), frm, eta=1e-6)
            mw = O.meir_wingreen(dev, [E], frm, eta=1e-6, scba_niter=0)
            J = _bond_currents(dev, E, outer)
            assert np.all(st == 0)
            assert np.abs(J - mw["curr"][0]).max() <= 1e-9 * max(1.0, np.abs(mw["curr"][0]).max())
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)
