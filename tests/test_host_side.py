"""Host side of the path: CSR -> blocks (extract_cont / zcsr2blk_sod), the
energy grid, fermi_f, integrate_el and the energy loop, checked against the
oracle's restatements (CPU) and, for the loop, the GPU engine (gpu)."""
import ctypes

import numpy as np
import pytest

from libnegf_b200 import energy as En
from libnegf_b200 import native
from libnegf_b200 import generators as G
from libnegf_b200 import structure as St
from oracle import oracle as O


def test_energy_grid_is_tunneling_int_def():
    E = En.energy_grid(-1.0, 1.0, 0.1)
    assert E.size == 21 and E[0] == -1.0 and abs(E[-1] - 1.0) < 1e-15
    assert En.energy_grid(0.0, 1.0, 0.3).size == 4          # nint(3.33) + 1
    assert En.local_points(10, 1, 3).tolist() == [1, 4, 7]


def test_fermi_matches_oracle():
    x = np.linspace(-2, 2, 101)
    for ef, kt in [(0.1, 0.02), (-0.3, 1e-3), (0.0, 0.0)]:
        ours = En.fermi_f(x, ef, kt)
        ref = np.array([O.fermi(v, ef, kt) for v in x])
        assert np.allclose(ours, ref, rtol=1e-15, atol=0)   # numpy's exp vs libm: 1 ulp


@pytest.mark.parametrize("mu1,mu2,kt1,kt2", [(-0.1, 0.1, 1e-3, 2e-3), (0.1, -0.05, 0.0, 3e-3), (0.0, 0.0, 1e-3, 1e-3)])
def test_integrate_el_matches_oracle(mu1, mu2, kt1, kt2):
    rng = np.random.default_rng(1)
    emin, emax, estep = -0.5, 0.5, 0.01
    T = rng.random(En.energy_grid(emin, emax, estep).size)
    a = En.integrate_el(T, mu1, mu2, kt1, kt2, emin, emax, estep)
    b = O.integrate_el(T, mu1, mu2, kt1, kt2, emin, emax, estep)
    assert abs(a - b) <= 1e-14 * max(1.0, abs(b))


def test_perfect_chain_current_is_window_times_gspin():
    """f90elph_deph-style known answer: T = 1 in the band, so the current is
    g_spin * (mu2 - mu1) for a bias window well inside the band."""
    emin, emax, estep = -1.0, 1.0, 0.01
    E = En.energy_grid(emin, emax, estep)
    T = np.ones((E.size, 1))
    I = En.electron_current(T, [(1, 2)], mu=[-0.2, 0.2], kT=[1e-4, 1e-4], emin=emin, emax=emax, estep=estep)
    assert abs(I[0] - 2.0 * 0.4) < 1e-6


@pytest.mark.parametrize("with_s", [False, True])
def test_csr_extraction_round_trip(with_s):
    dev = G.transport_c1(nbl=4, n=6, seed=2, density=0.5) if with_s else G.transport_c0(nbl=5, n=4, seed=3)
    H, S, plend, cblk, ss, se, ce = St.csr_from_device(dev)
    d2 = St.device_from_csr(H, S, plend, cblk, ss, se, ce)
    for name in ("h_diag", "h_upper", "h_lower", "lead_h00", "lead_h01", "hmc"):
        for a, b in zip(getattr(dev, name), getattr(d2, name)):
            assert np.array_equal(a, b)
    E = np.linspace(-1, 1, 7)
    t1, _, _ = O.transmission(dev, E, eta=1e-6)
    t2, _, _ = O.transmission(d2, E, eta=1e-6)
    assert np.array_equal(t1, t2)


@pytest.mark.parametrize("with_s", [False, True])
def test_csr_arrays_hold_h_and_s_on_one_pattern(with_s):
    """The 1-based arrays of negf_b200_upload_csr rebuild H and S exactly."""
    import scipy.sparse as sp
    dev = G.transport_c1(nbl=4, n=6, seed=2, density=0.5) if with_s else G.transport_c0(nbl=5, n=4, seed=3)
    H, S, *_ = St.csr_from_device(dev)
    rp, ci, hv, sv = St.csr_arrays(H, S)
    assert rp.dtype == np.int32 and ci.dtype == np.int32 and rp[0] == 1 and rp[-1] == ci.size + 1
    n = rp.size - 1
    H2 = sp.csr_matrix((hv, ci - 1, rp - 1), shape=(n, n))
    assert abs(H2 - sp.csr_matrix(H)).max() == 0
    if with_s:
        S2 = sp.csr_matrix((sv, ci - 1, rp - 1), shape=(n, n))
        assert abs(S2 - sp.csr_matrix(S)).max() == 0
    else:
        assert sv is None


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["c0", "c1_S", "three"])
def test_upload_csr_matches_block_upload(gpu_ctx, case):
    """Blocks extracted from the CSR on the GPU give the same T and DOS, bit
    for bit, as the host-extracted blocks."""
    dev = {"c0": lambda: G.transport_c0(nbl=5, n=12, seed=3),
           "c1_S": lambda: G.transport_c1(nbl=4, n=20, seed=2, density=0.3),
           "three": lambda: G.transport_c0(nbl=5, n=8, seed=1, cblk=[1, 5, 3])}[case]()
    H, S, plend, cblk, ss, se, ce = St.csr_from_device(dev)
    E = np.linspace(-2, 2, 9)
    d1 = gpu_ctx.upload(dev)
    d2 = gpu_ctx.upload_csr(H, S, plend, cblk, ss, se, ce)
    try:
        pairs = [(1, 2), (1, 3), (2, 3)] if case == "three" else [(1, 2)]
        T1, l1, _, _ = gpu_ctx.transmissions(d1, E, pairs, eta=1e-4)
        T2, l2, _, _ = gpu_ctx.transmissions(d2, E, pairs, eta=1e-4)
        assert np.array_equal(T1, T2)
        if case != "three":
            _, dos1, _, _ = gpu_ctx.transmission_dos(d1, E, eta=1e-4)
            _, dos2, _, _ = gpu_ctx.transmission_dos(d2, E, eta=1e-4)
            assert np.array_equal(dos1, dos2)
        # a column index outside the matrix is an argument error, not a fault
        rp, ci, hv, sv = St.csr_arrays(H, S)
        ci[3] = rp.size + 5
        L = native.load()
        a = lambda x: np.ascontiguousarray(x, dtype=np.int32)
        dp = lambda x: x.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if x is not None else None
        ip = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        did = ctypes.c_int32()
        pe, cb, s1, s2, c2 = a(plend), a(cblk), a(ss), a(se), a(ce)
        rc = L.negf_b200_upload_csr(gpu_ctx.handle, rp.size - 1, ci.size, ip(rp), ip(ci), dp(hv), dp(sv), pe.size,
                                    ip(pe), cb.size, ip(cb), ip(s1), ip(s2), ip(c2), ctypes.byref(did))
        assert rc == native.BAD_ARG
    finally:
        gpu_ctx.release(d1)
        gpu_ctx.release(d2)


@pytest.mark.parametrize("gen", ["c0", "c1_S"])
def test_bound_surface_known_answer(gen):
    """surfdim > 0 (src/contselfenergy.F90:226-243): surface orbitals that are
    periodic copies of the lead PL leave every result unchanged, through the
    oracle, its long-double path and the NumPy twin; the CSR round trip with
    surface orbitals (negf_init_structure's surfstart/surfend) is exact."""
    from oracle import twin as TW
    dev0 = (G.transport_c0(nbl=5, n=8, seed=4) if gen == "c0"
            else G.transport_c1(nbl=4, n=10, seed=4, density=0.3))
    dev = G.with_periodic_surface(G.with_periodic_surface(dev0, 0, 1), 1, 2)
    assert dev.surf_size == [dev0.lead_size[0], 2 * dev0.lead_size[1]]
    E = np.linspace(-1.5, 1.5, 9)
    T0 = O.transmission(dev0, E, eta=1e-4)[0]
    T, nc, st = O.transmission(dev, E, eta=1e-4)
    assert np.all(st == 0)
    assert np.all(np.abs(T - T0) <= np.maximum(1e-10 * np.abs(T0), 1e-11))
    Tx = O.transmission_xp(dev, E, eta=1e-4)[0]
    assert np.all(np.abs(Tx - T) <= np.maximum(1e-10 * np.abs(T), 1e-12))
    Tt = np.array([TW.point_transmission(dev, e, eta=1e-4)[0] for e in E], dtype=float)
    assert np.all(np.abs(Tt - T) <= np.maximum(1e-10 * np.abs(T), 1e-12))
    H, S, plend, cblk, ss, se, ce = St.csr_from_device(dev)
    assert [e - s + 1 for s, e in zip(ss, se)] == dev.surf_size
    back = St.device_from_csr(H, S, plend, cblk, ss, se, ce)
    assert np.array_equal(O.transmission(back, E, eta=1e-4)[0], T)


@pytest.mark.gpu
def test_tunneling_and_dos_loop_matches_oracle(gpu_ctx):
    """tunn_mat over two k-points with weights, and the Landauer current."""
    devs = [G.transport_c0(nbl=5, n=6, seed=s) for s in (0, 1)]
    w = [0.25, 0.75]
    ids = [gpu_ctx.upload(d) for d in devs]
    try:
        emin, emax, estep = -2.0, 2.0, 0.05
        E, tunn, _, st = En.tunneling_and_dos(gpu_ctx, ids, w, emin, emax, estep, [(1, 2)], eta=1e-4)
        ref = sum(O.transmission(d, E, eta=1e-4)[0] * wk for d, wk in zip(devs, w))
        assert np.all(st == 0)
        assert np.abs(tunn[:, 0] - ref).max() <= 1e-9 * max(1.0, np.abs(ref).max())
        I = En.electron_current(tunn, [(1, 2)], mu=[-0.1, 0.1], kT=[1e-3, 1e-3], emin=emin, emax=emax, estep=estep)
        Iref = O.integrate_el(ref, -0.1, 0.1, 1e-3, 1e-3, emin, emax, estep) * 2.0
        assert abs(I[0] - Iref) <= 1e-9 * max(1.0, abs(Iref))
    finally:
        for i in ids:
            gpu_ctx.release(i)
