"""The CPU oracle pinned against known answers (no GPU).

The reference's golden T(E) files are git-LFS pointers absent from the
reference tree, so the oracle is pinned by: the perfect-chain transmission
(T = 1 in band), the closed-form surface Green's function of a semi-infinite
chain, the two current checks of tests/f90elph_deph/hello.F90:88-119
(zero coupling -> current 2.0 +- 1e-4; coupling 0.05 -> [1.90, 1.95]), the
identities of the non-equilibrium solve (current conservation, flat layer
current) and an independent NumPy twin.
"""
import numpy as np
import pytest

from libnegf_b200 import generators as G
from oracle import oracle as O
from oracle import twin as TW
from conftest import assert_T_close


@pytest.mark.parametrize("m,nbl,cblk", [(1, 1, None), (1, 4, None), (3, 4, None), (3, 4, [4, 1]), (2, 2, None)])
def test_chain_transmission_is_one_in_band(m, nbl, cblk):
    dev = G.chain(n_per_pl=m, nbl=nbl, cblk=cblk)
    E = np.linspace(-1.9, 1.9, 11)
    T, ncyc, st = O.transmission(dev, E, eta=1e-6, sgf_tol=1e-12)
    assert np.all(st == 0)
    np.testing.assert_allclose(T, 1.0, atol=1e-8)
    # outside the band: evanescent, T ~ 0
    T2, _, _ = O.transmission(dev, np.array([2.5, -3.0]), eta=1e-6)
    assert np.all(T2 < 1e-6)


def _ladder(nbl=5, t=1.0, tperp=0.5):
    """Perfect two-leg ladder, one rung per PL: H00 = [[0, -tp], [-tp, 0]],
    rung-to-rung hopping -t on both legs.  Bands +-tp - 2t cos k."""
    from libnegf_b200.device import Device
    H0 = np.array([[0.0, -tperp], [-tperp, 0.0]], dtype=np.complex128)
    V = -t * np.eye(2, dtype=np.complex128)
    return Device([H0.copy() for _ in range(nbl)], [V.copy() for _ in range(nbl - 1)],
                  [V.copy() for _ in range(nbl - 1)], [1, nbl], [H0.copy(), H0.copy()], [V.copy(), V.copy()],
                  [V.copy(), V.copy()])


def test_ladder_transmission_counts_open_channels():
    """Known answer with two orbitals per PL: a perfect ladder transmits one
    unit per open band, T(E) = #{s = +-1 : |E - s tp| < 2t} (2 in the
    middle, 1 where only one band is open, 0 outside)."""
    dev = _ladder()
    E = np.array([-2.3, -1.8, -1.0, -0.2, 0.4, 1.2, 1.9, 2.2, 2.7])
    expect = np.array([sum(abs(e - s * 0.5) < 2.0 for s in (1, -1)) for e in E], dtype=float)
    T, nc, st = O.transmission(dev, E, eta=1e-7)
    assert np.all(st == 0)
    assert np.abs(T - expect).max() < 1e-4


@pytest.mark.parametrize("e", [-1.7, -0.3, 0.0, 0.9, 1.95, 2.4, -3.0])
def test_surface_green_closed_form(e):
    t = 1.0
    Ec = e + 1e-6j
    g, ncyc, st = O.decimation(np.array([[Ec]]), np.array([[t]]), np.array([[t]]), tol=1e-12)
    r = np.sqrt(Ec * Ec - 4 * t * t + 0j)
    cands = [(Ec - r) / (2 * t * t), (Ec + r) / (2 * t * t)]
    ga = [c for c in cands if c.imag <= 0 and abs(c) <= 1 / t + 1e-9]
    ga = min(ga, key=lambda c: abs(c))
    assert st == 0
    # E = 0 is the band centre, where the first decimation step inverts
    # Ao = i*eta; there the iteration lands within ~1e-4 of the closed form
    tol = 1e-4 if e == 0.0 else 1e-9
    assert abs(g[0, 0] - ga) < tol * max(1.0, abs(ga))


def test_decimation_matches_twin():
    rng = np.random.default_rng(5)
    n = 6
    H0 = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    H0 = (H0 + H0.conj().T) / 2
    V = 0.4 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    Ec = 0.3 + 1e-6j
    Ao, Bo, Co = Ec * np.eye(n) - H0, -V, -V.conj().T
    g, nc, st = O.decimation(Ao, Bo, Co)
    g2, nc2 = TW.decimation(Ao, Bo, Co)
    assert nc == nc2
    assert np.abs(g - g2).max() < 1e-10 * np.abs(g2).max()


def test_zinv_is_inverse():
    rng = np.random.default_rng(1)
    A = rng.standard_normal((9, 9)) + 1j * rng.standard_normal((9, 9))
    X, st = O.zinv(A)
    assert st == 0
    assert np.abs(A @ X - np.eye(9)).max() < 1e-12


@pytest.mark.parametrize("gen", ["c0", "c1s", "uneven", "ncont", "rev"])
def test_transmission_matches_twin(gen):
    if gen == "c0":
        dev = G.transport_c0(nbl=6, n=8, seed=0)
        E = np.linspace(-3, 3, 13)
    elif gen == "c1s":
        dev = G.transport_c1(nbl=5, n=12, seed=2, density=0.3)
        E = np.linspace(-2, 2, 9)
    elif gen == "uneven":
        dev = G.uneven([5, 7, 3, 6], seed=4)
        E = np.linspace(-2, 2, 9)
    elif gen == "ncont":
        dev = G.transport_c0(nbl=6, n=8, seed=1, cblk=[2, 5])
        E = np.linspace(-3, 3, 13)
    else:
        dev = G.transport_c0(nbl=5, n=6, seed=3, cblk=[5, 1])
        E = np.linspace(-3, 3, 13)
    T, ncyc, st = O.transmission(dev, E, eta=1e-6)
    Tt = np.array([TW.point_transmission(dev, e, eta=1e-6)[0] for e in E])
    assert_T_close(T, Tt, rtol=1e-9, atol=1e-13)


def test_dos_matches_twin():
    dev = G.transport_c0(nbl=5, n=6, seed=2)
    E = np.linspace(-3, 3, 7)
    T, dos, nc, st = O.transmission_dos(dev, E, eta=1e-6, dos_delta=1e-4)
    for k, e in enumerate(E):
        t2, d2 = TW.point_dos(dev, e, eta=1e-6, dos_delta=1e-4)
        assert abs(T[k] - t2) <= 1e-10 * max(1e-6, abs(t2)) + 1e-13
        assert np.abs(dos[k] - d2).max() <= 1e-10 * max(1.0, np.abs(d2).max())


def test_dos_sum_rule_chain():
    """-Im Gr/pi of a perfect chain site = 1/(pi sqrt(4t^2 - E^2)) in band."""
    dev = G.chain(n_per_pl=2, nbl=3)
    E = np.array([-1.0, 0.0, 0.5])
    T, dos, _, _ = O.transmission_dos(dev, E, eta=1e-7, dos_delta=1e-7)
    expect = 1.0 / (np.pi * np.sqrt(4.0 - E * E))
    np.testing.assert_allclose(dos, np.repeat(expect[:, None], dos.shape[1], axis=1), rtol=1e-5)


def _elph_chain():
    # tests/f90elph_deph: 60-orbital device in 6 PLs of 10, contacts of 20,
    # cblk = [6, 1], mu = -0.5 / 0.5, kT = 1e-3, E in [-2, 2] step 0.1
    return G.chain(n_per_pl=10, nbl=6, cblk=[6, 1])


def test_elph_deph_zero_coupling_current():
    dev = _elph_chain()
    E = np.arange(-2.0, 2.0 + 1e-9, 0.1)
    res = O.meir_wingreen(dev, E, frm=[1.0, 0.0], coupling=np.zeros(60), eta=1e-4, scba_niter=5)
    cur = O.integrate_el(res["curr"][:, 0], -0.5, 0.5, 1e-3, 1e-3, -2.0, 2.0, 0.1) * 2.0
    assert abs(cur - 2.0) < 1e-4
    assert np.all(res["scba_iter"] == 2)


def test_elph_deph_finite_coupling_current():
    dev = _elph_chain()
    E = np.arange(-2.0, 2.0 + 1e-9, 0.1)
    res = O.meir_wingreen(dev, E, frm=[1.0, 0.0], coupling=np.full(60, 0.05), eta=1e-4, scba_niter=5)
    cur = abs(O.integrate_el(res["curr"][:, 0], -0.5, 0.5, 1e-3, 1e-3, -2.0, 2.0, 0.1) * 2.0)
    assert 1.90 <= cur <= 1.95
    # coherent current is larger (dephasing reduces it)
    # current conservation I_1 = -I_2 and a flat layer-current profile
    # (at SCBA-converged points; the band edges stop at scba_niter)
    ok = res["scba_err"] < 1e-6
    assert ok.sum() >= 30
    np.testing.assert_allclose(res["curr"][ok, 0], -res["curr"][ok, 1], atol=1e-6)
    lc = res["layer_curr"][ok]
    np.testing.assert_allclose(lc, np.repeat(lc[:, :1], lc.shape[1], axis=1), atol=1e-6)


def test_fermi_and_integrate_el():
    assert O.fermi(0.0, 0.0, 0.1) == 0.5
    assert O.fermi(1.0, 0.0, 0.0) == 0.0 and O.fermi(-1.0, 0.0, 0.0) == 1.0
    # constant T = 1 over a window much wider than mu2 - mu1 -> current = mu2 - mu1
    E = np.linspace(-2, 2, 41)
    cur = O.integrate_el(np.ones_like(E), -0.3, 0.2, 1e-3, 1e-3, -2.0, 2.0, 0.1)
    assert abs(cur - 0.5) < 1e-6
    assert abs(O.integrate_el(np.ones_like(E), 0.2, -0.3, 1e-3, 1e-3, -2.0, 2.0, 0.1) + 0.5) < 1e-6


def _scba_case():
    from libnegf_b200.energy import fermi_f
    dev = G.transport_c0(nbl=8, n=12, seed=0)
    E = np.linspace(-1.0, 1.0, 13)
    kT = 8.617333262e-5 * 300.0
    frm = np.stack([fermi_f(E, 0.1, kT), fermi_f(E, -0.1, kT)], axis=1)
    return dev, E, frm, np.full(dev.norb, 0.1)


def test_scba_mix_one_is_the_reference_rule():
    dev, E, frm, cpl = _scba_case()
    a = O.meir_wingreen(dev, E, frm, coupling=cpl, eta=1e-4, scba_niter=30)
    b = O.meir_wingreen(dev, E, frm, coupling=cpl, eta=1e-4, scba_niter=30, scba_mix=1.0, scba_rule=0)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_scba_mixing_and_current_rule_reach_the_same_fixed_point():
    """Linear mixing changes the path, not the SCBA fixed point.  The current
    rule stops once the contact-1 current moves by less than the tolerance:
    the currents agree with the converged ones, the densities need not (where
    both contacts are filled the current is ~0 from the first sweep on)."""
    dev, E, frm, cpl = _scba_case()
    ref = O.meir_wingreen(dev, E, frm, coupling=cpl, eta=1e-4, scba_niter=200, scba_tol=1e-12)
    mix = O.meir_wingreen(dev, E, frm, coupling=cpl, eta=1e-4, scba_niter=200, scba_tol=1e-12, scba_mix=0.5)
    ok = (ref["scba_err"] < 1e-12) & (mix["scba_err"] < 1e-12)
    assert ok.sum() >= 10
    scale = np.abs(ref["curr"]).max()
    assert np.abs(mix["curr"][ok] - ref["curr"][ok]).max() <= 1e-8 * scale
    assert np.abs(mix["layer_dens"][ok] - ref["layer_dens"][ok]).max() <= 1e-8 * np.abs(ref["layer_dens"]).max()
    cur = O.meir_wingreen(dev, E, frm, coupling=cpl, eta=1e-4, scba_niter=200, scba_tol=1e-11, scba_mix=0.5,
                          scba_rule=1)
    ok = (ref["scba_err"] < 1e-12) & (cur["scba_err"] < 1e-11)
    assert ok.sum() >= 10 and np.all(cur["scba_iter"] >= 2)
    assert np.abs(cur["curr"][ok] - ref["curr"][ok]).max() <= 1e-8 * scale
