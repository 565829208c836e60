"""GPU parity: the CUDA path (through the C-ABI) against the CPU oracle on
the same seeded inputs.

Bound: |T - T_oracle| <= max(1e-10 |T_oracle|, 1e-13), strict at every point
where three CPU FP64 paths of the algorithm (the oracle's and two restated
ones) all lie within an eighth of it from the long-double solution; the
decimation's iteration count equals the oracle's at every point.  At the
other points (ill-conditioned device solves: the device blocks carry no
broadening) the GPU result must lie as close to the long-double solution as
the CPU FP64 paths do (conftest.assert_parity)."""
import ctypes

import numpy as np
import pytest

from libnegf_b200 import generators as G
from libnegf_b200 import native
from oracle import oracle as O
from conftest import assert_parity, assert_T_strict, oracle_spread, xp_reference

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _rand(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _dev(a):
    """complex128 numpy (column-major semantics) -> device tensor of the
    Fortran-ordered data"""
    flat = np.ascontiguousarray(np.asarray(a, dtype=np.complex128).reshape(a.shape[0], -1, a.shape[-1])
                                .transpose(0, 2, 1))   # batch x cols x rows == column-major per item
    return torch.from_numpy(flat).cuda()


def _host(t, rows, cols):
    return t.cpu().numpy().transpose(0, 2, 1).reshape(-1, rows, cols)


@pytest.mark.parametrize("m,n,k,dagger", [(1, 1, 1, 0), (8, 8, 8, 0), (32, 32, 32, 0), (64, 64, 64, 0),
                                          (17, 33, 65, 0), (130, 70, 100, 0), (48, 40, 24, 1), (48, 40, 24, 2),
                                          (256, 256, 256, 0), (100, 100, 100, 2)])
def test_zgemm_batched(m, n, k, dagger):
    rng = np.random.default_rng(m * 1000 + n * 10 + k + dagger)
    b = 3
    A = _rand(rng, (b, k, m)) if dagger == 1 else _rand(rng, (b, m, k))
    B = _rand(rng, (b, n, k)) if dagger == 2 else _rand(rng, (b, k, n))
    C = _rand(rng, (b, m, n))
    alpha, beta = np.array([0.7, -0.3]), np.array([0.25, 0.5])
    dA, dB, dC = _dev(A), _dev(B), _dev(C)
    L = native.load()
    dp = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    rc = L.negf_b200_zgemm_batched(b, m, n, k, dp(alpha), dA.data_ptr(), 2 * A[0].size, dB.data_ptr(),
                                   2 * B[0].size, dp(beta), dC.data_ptr(), 2 * m * n, dagger, None)
    torch.cuda.synchronize()
    assert rc == 0
    opA = A.conj().transpose(0, 2, 1) if dagger == 1 else A
    opB = B.conj().transpose(0, 2, 1) if dagger == 2 else B
    ref = (0.7 - 0.3j) * (opA @ opB) + (0.25 + 0.5j) * C
    got = _host(dC, m, n)
    assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max()) * np.sqrt(k)


@pytest.mark.parametrize("n", [24, 96, 256, 512])
def test_zinv_residual_on_nearly_singular_matrices(n):
    """Gauss-Jordan is not backward stable: on a matrix with condition number
    1e9-1e11 its residual A X - I can reach 1e-5 .. 1e-4 where an LU inverse
    stays at 1e-10.  The residual probe and its Newton steps bring it below
    1e-5 (or to 100x the LU residual), the forward error within cond * eps."""
    rng = np.random.default_rng(100 + n)
    b = 3
    A = np.empty((b, n, n), dtype=np.complex128)
    for i, c in enumerate((1e9, 1e10, 1e11)):
        U = np.linalg.qr(_rand(rng, (n, n)))[0]
        V = np.linalg.qr(_rand(rng, (n, n)))[0]
        A[i] = (U * np.geomspace(1.0, 1.0 / c, n)) @ V
    dA = _dev(A)
    dX = torch.empty_like(dA)
    info = torch.zeros(b, dtype=torch.int32, device="cuda")
    L = native.load()
    work = torch.empty(L.negf_b200_zinv_work_bytes(b, n), dtype=torch.uint8, device="cuda")
    rc = L.negf_b200_zinv_batched(b, n, dA.data_ptr(), dX.data_ptr(), info.data_ptr(), work.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0 and int(info.abs().sum()) == 0
    X = _host(dX, n, n)
    for i in range(b):
        Xr = np.linalg.inv(A[i])
        res = np.abs(A[i] @ X[i] - np.eye(n)).max()
        res_lu = np.abs(A[i] @ Xr - np.eye(n)).max()
        assert res <= max(100 * res_lu, 1e-5), (i, res, res_lu)     # refined above a probe of 1e-5
        cond = np.linalg.cond(A[i])
        assert np.abs(X[i] - Xr).max() <= 1e-14 * cond * np.abs(Xr).max() * n


@pytest.mark.parametrize("n", [1, 2, 5, 16, 33, 64, 65, 100, 128, 200, 256, 257, 512, 513, 777, 1024])
def test_zinv_batched(n):
    rng = np.random.default_rng(n)
    b = 2
    A = _rand(rng, (b, n, n)) + 2.0 * np.sqrt(n) * np.eye(n) * (rng.random() < 2)
    A[1] = _rand(rng, (n, n))   # general (pivoting exercised)
    dA = _dev(A)
    dX = torch.empty_like(dA)
    info = torch.zeros(b, dtype=torch.int32, device="cuda")
    L = native.load()
    wb = L.negf_b200_zinv_work_bytes(b, n)
    work = torch.empty(max(wb, 16), dtype=torch.uint8, device="cuda")
    rc = L.negf_b200_zinv_batched(b, n, dA.data_ptr(), dX.data_ptr(), info.data_ptr(), work.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0 and int(info.abs().sum()) == 0
    X = _host(dX, n, n)
    for i in range(b):
        Xr = np.linalg.inv(A[i])
        cond = np.linalg.cond(A[i])
        assert np.abs(X[i] - Xr).max() <= 1e-14 * cond * max(1.0, np.abs(Xr).max()) * n


def test_zinv_singular_reports_info():
    n = 8
    A = np.eye(n, dtype=np.complex128)[None]
    A[0, 3, 3] = 0.0
    dA = _dev(A)
    dX = torch.empty_like(dA)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    L = native.load()
    rc = L.negf_b200_zinv_batched(1, n, dA.data_ptr(), dX.data_ptr(), info.data_ptr(), None, None)
    torch.cuda.synchronize()
    assert rc == 0 and int(info[0]) == 4


@pytest.mark.parametrize("n", [1, 4, 32, 80])
def test_decimation_batched(n):
    dev = G.transport_c0(nbl=3, n=n, seed=n)
    Es = [-1.3, 0.2, 2.2]
    b = len(Es)
    Ao, Bo, Co = [], [], []
    for e in Es:
        Ec = e + 1e-6j
        Ao.append(Ec * np.eye(n) - dev.lead_h00[1])
        Bo.append(-dev.lead_h01[1])
        Co.append(-dev.lead_h01[1].conj().T)
    Ao, Bo, Co = np.array(Ao), np.array(Bo), np.array(Co)
    dAo, dBo, dCo = _dev(Ao), _dev(Bo), _dev(Co)
    dG = torch.empty_like(dAo)
    ncyc = torch.zeros(b, dtype=torch.int32, device="cuda")
    L = native.load()
    work = torch.empty(L.negf_b200_decimation_work_bytes(b, n), dtype=torch.uint8, device="cuda")
    rc = L.negf_b200_decimation_batched(b, n, dAo.data_ptr(), dBo.data_ptr(), dCo.data_ptr(), dG.data_ptr(),
                                        ncyc.data_ptr(), 1e-9, 300, work.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    Gd = _host(dG, n, n)
    for i in range(b):
        g, nc, st = O.decimation(Ao[i], Bo[i], Co[i], tol=1e-9)
        assert int(ncyc[i]) == nc
        gx = O.decimation_xp(Ao[i], Bo[i], Co[i], tol=1e-9)[0]
        gd = O.decimation_xp(Ao[i], Bo[i], Co[i], tol=1e-9, extended=False)[0]
        gg = O.decimation_xp(Ao[i], Bo[i], Co[i], tol=1e-9, extended=False, gauss_jordan=True)[0]
        bound = 1e-10 * max(1.0, np.abs(g).max())
        for part in (np.real, np.imag):
            assert_parity(part(Gd[i]), part(g), bound, ref_x=part(gx), others=(part(gd), part(gg)),
                          what="surface GF (n=%d, E=%g)" % (n, Es[i]))


CASES = {
    "chain1": lambda: (G.chain(1, 4), np.linspace(-1.9, 1.9, 9)),
    "chain3_rev": lambda: (G.chain(3, 5, cblk=[5, 1]), np.linspace(-1.9, 1.9, 9)),
    "nbl1": lambda: (G.transport_c0(nbl=1, n=6, seed=1), np.linspace(-3, 3, 9)),
    "nbl2": lambda: (G.transport_c0(nbl=2, n=6, seed=1), np.linspace(-3, 3, 9)),
    "c0_small": lambda: (G.transport_c0(nbl=6, n=8, seed=0), np.linspace(-3, 3, 17)),
    "c0_n32": lambda: (G.transport_c0(nbl=20, n=32, seed=0), G.energy_grid(-3, 3, 512)[::16]),
    "c1_S": lambda: (G.transport_c1(nbl=5, n=12, seed=2, density=0.3), np.linspace(-2, 2, 9)),
    "uneven": lambda: (G.uneven([5, 7, 3, 6], seed=4), np.linspace(-2, 2, 9)),
    "ncont": lambda: (G.transport_c0(nbl=6, n=8, seed=1, cblk=[2, 5]), np.linspace(-3, 3, 13)),
    "n80": lambda: (G.transport_c0(nbl=4, n=80, seed=6), np.linspace(-3, 3, 5)),
    "n130_S": lambda: (G.transport_c1(nbl=3, n=130, seed=7, density=0.1), np.linspace(-2, 2, 3)),
}


def _o_T(E, **kw):
    def run(d):
        T, nc, st = O.transmission(d, E, **kw)
        return {"T": T, "ncyc": nc, "status": st}
    return run


def _o_dos(E, **kw):
    def run(d):
        T, dos, nc, st = O.transmission_dos(d, E, **kw)
        return {"T": T, "dos": dos, "ncyc": nc, "status": st}
    return run


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("case", sorted(CASES))
def test_transmission_parity(gpu_ctx, case, schedule):
    """schedule 0: lock step where the call fits it (2 contacts on blocks 1
    and nbl, one PL size n <= 32), else the engine; schedule 1: the engine."""
    dev, E = CASES[case]()
    did = gpu_ctx.upload(dev)
    gpu_ctx.set_options(schedule=schedule)
    try:
        T, ncyc, st = gpu_ctx.transmission(did, E, eta=1e-6)
        ref, spread = oracle_spread(_o_T(E, eta=1e-6), dev, nsamp=2)
        assert np.all(st == ref["status"])
        assert np.array_equal(ncyc, ref["ncyc"])
        assert_T_strict(T, ref["T"], xp_reference(dev, E, 1e-6), spread=spread["T"])
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)


@pytest.mark.parametrize("gen", ["c0", "c1_S"])
def test_transmission_parity_band_edges(gpu_ctx, gen):
    """64 energies within 1e-3 eV of the band edges of lead 1 (the cluster of
    the 512-orbital mixed-precision config), eta = 1e-6, where the solve is
    least well conditioned."""
    dev = (G.transport_c0(nbl=6, n=16, seed=5) if gen == "c0"
           else G.transport_c1(nbl=5, n=24, seed=3, density=0.2))
    E = G.band_edge_energies(dev, contact=0, nk=64, n_edges=64, window=1e-3)
    did = gpu_ctx.upload(dev)
    try:
        T, ncyc, st = gpu_ctx.transmission(did, E, eta=1e-6, check=False)
        ref, spread = oracle_spread(_o_T(E, eta=1e-6), dev, nsamp=2)
        assert np.all(st == ref["status"])
        assert np.array_equal(ncyc, ref["ncyc"])
        assert_T_strict(T, ref["T"], xp_reference(dev, E, 1e-6), spread=spread["T"])
    finally:
        gpu_ctx.release(did)


@pytest.mark.parametrize("case", ["chain1", "c0_small", "c0_n32"])
def test_transmission_parity_default_eta(gpu_ctx, case):
    """At libNEGF's default broadening delta = 1e-4 (lib_param.F90:628)."""
    dev, E = CASES[case]()
    did = gpu_ctx.upload(dev)
    try:
        T, ncyc, st = gpu_ctx.transmission(did, E, eta=1e-4)
        ref, spread = oracle_spread(_o_T(E, eta=1e-4), dev, nsamp=2)
        assert np.all(st == ref["status"])
        assert np.array_equal(ncyc, ref["ncyc"])
        assert_T_strict(T, ref["T"], xp_reference(dev, E, 1e-4), spread=spread["T"])
    finally:
        gpu_ctx.release(did)


@pytest.mark.parametrize("case", ["chain3_rev", "c0_small", "c1_S", "uneven", "ncont", "n80"])
def test_transmission_dos_parity(gpu_ctx, case):
    dev, E = CASES[case]()
    did = gpu_ctx.upload(dev)
    try:
        T, dos, ncyc, st = gpu_ctx.transmission_dos(did, E, eta=1e-6, dos_delta=1e-4)
        ref, spread = oracle_spread(_o_dos(E, eta=1e-6, dos_delta=1e-4), dev, nsamp=2)
        assert np.all(st == ref["status"])
        assert np.array_equal(ncyc, ref["ncyc"])
        x = xp_reference(dev, E, 1e-6, dos_delta=1e-4)
        assert_T_strict(T, ref["T"], x, spread=spread["T"])
        # DOS: 1e-10 relative to the largest entry
        bound = 1e-10 * max(np.abs(ref["dos"]).max(), 1.0)
        assert_parity(dos, ref["dos"], bound, ref_x=None if x is None else x["dos_x"],
                      others=() if x is None else (x["dos_d"], x["dos_g"]), spread=spread["dos"], what="DOS",
                      rows=True)
    finally:
        gpu_ctx.release(did)


def test_multi_device_batch(gpu_ctx):
    """Points of different devices (k-points / requests) in one launch."""
    d1, E1 = CASES["c0_small"]()
    d2, E2 = CASES["uneven"]()
    i1, i2 = gpu_ctx.upload(d1), gpu_ctx.upload(d2)
    try:
        ids = np.array([i1] * len(E1) + [i2] * len(E2), dtype=np.int32)
        E = np.concatenate([E1, E2])
        T, nc, st = gpu_ctx.transmission(ids, E, eta=1e-6)
        r1, s1 = oracle_spread(_o_T(E1, eta=1e-6), d1, nsamp=2)
        r2, s2 = oracle_spread(_o_T(E2, eta=1e-6), d2, nsamp=2)
        assert np.array_equal(nc, np.concatenate([r1["ncyc"], r2["ncyc"]]))
        assert_T_strict(T[:len(E1)], r1["T"], xp_reference(d1, E1, 1e-6), spread=s1["T"])
        assert_T_strict(T[len(E1):], r2["T"], xp_reference(d2, E2, 1e-6), spread=s2["T"])
    finally:
        gpu_ctx.release(i1)
        gpu_ctx.release(i2)


@pytest.mark.parametrize("case", ["elph", "c0_deph", "c1_S_deph", "c0_mix_current_rule", "c1_S_mix"])
def test_meir_wingreen_parity(gpu_ctx, case):
    mix, rule, niter, tol = 1.0, 0, 5, 1e-7
    if case == "elph":
        dev = G.chain(10, 6, cblk=[6, 1])
        E = np.arange(-2.0, 2.0 + 1e-9, 0.1)
        cpl = np.full(dev.norb, 0.05)
        frm = [1.0, 0.0]
    elif case == "c0_deph":
        dev = G.transport_c0(nbl=5, n=8, seed=3)
        E = np.linspace(-1, 1, 7)
        cpl = np.full(dev.norb, 0.1)
        frm = np.stack([[0.9, 0.2]] * len(E))
    elif case == "c0_mix_current_rule":
        # the elastic-dephasing workload's rule: mixing 0.5, stop on a current change below 1e-8
        dev = G.transport_c0(nbl=6, n=8, seed=3)
        E = np.linspace(-1, 1, 9)
        cpl = np.full(dev.norb, 0.1)
        frm = np.stack([[0.9, 0.2]] * len(E))
        mix, rule, niter, tol = 0.5, 1, 40, 1e-8
    elif case == "c1_S_mix":
        dev = G.transport_c1(nbl=4, n=10, seed=4, density=0.3)
        E = np.linspace(-1, 1, 5)
        cpl = np.full(dev.norb, 0.1)
        frm = [1.0, 0.0]
        mix, niter = 0.3, 8
    else:
        dev = G.transport_c1(nbl=4, n=10, seed=4, density=0.3)
        E = np.linspace(-1, 1, 5)
        cpl = np.full(dev.norb, 0.1)
        frm = [1.0, 0.0]
    did = gpu_ctx.upload(dev)
    gpu_ctx.set_options(scba_niter=niter, scba_tol=tol, scba_mix=mix, scba_rule=rule)
    try:
        r = gpu_ctx.meir_wingreen(did, E, frm, coupling=cpl, eta=1e-4)
        o, spread = oracle_spread(lambda d: O.meir_wingreen(d, E, frm, coupling=cpl, eta=1e-4, scba_niter=niter,
                                                            scba_tol=tol, scba_mix=mix, scba_rule=rule), dev,
                                  nsamp=2)
        assert np.all(r["status"] == o["status"])
        assert np.array_equal(r["scba_iter"], o["scba_iter"])
        assert np.array_equal(r["ncyc"], o["ncyc"])
        for key in ("curr", "layer_curr", "layer_dens"):
            a, b = r[key], o[key]
            bound = 1e-10 * max(1.0, np.abs(b).max())
            assert_parity(a, b, bound, spread=spread[key], what=key)
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)


def test_meir_wingreen_dev_matches_host_call(gpu_ctx):
    """negf_b200_meir_wingreen_dev (device buffers, caller's stream) gives the
    host-buffer call's outputs bit for bit."""
    dev = G.transport_c0(nbl=5, n=8, seed=3)
    E = np.linspace(-1, 1, 7)
    cpl = np.full(dev.norb, 0.1)
    frm = np.ascontiguousarray(np.stack([[0.9, 0.2]] * len(E)))
    did = gpu_ctx.upload(dev)
    gpu_ctx.set_options(scba_niter=6, scba_mix=0.5, scba_rule=1, scba_tol=1e-8)
    try:
        r = gpu_ctx.meir_wingreen(did, E, frm, coupling=cpl, eta=1e-4)
        n, nbl, ncs = len(E), dev.nbl, 3      # strides above the minimum
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        d_ids, d_E = t(np.full(n, did, dtype=np.int32)), t(E)
        d_frm = t(np.concatenate([frm, np.zeros((n, 1))], axis=1))
        d_cpl = t(cpl)
        d_curr = torch.zeros((n, ncs), dtype=torch.float64, device="cuda")
        d_lc = torch.zeros((n, nbl + 1), dtype=torch.float64, device="cuda")
        d_ld = torch.zeros((n, nbl + 1), dtype=torch.float64, device="cuda")
        d_it = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_err = torch.zeros(n, dtype=torch.float64, device="cuda")
        d_nc = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_st = torch.zeros(n, dtype=torch.int32, device="cuda")
        s = torch.cuda.Stream()
        L = native.load()
        rc = L.negf_b200_meir_wingreen_dev(gpu_ctx.handle, n, d_ids.data_ptr(), d_E.data_ptr(), 1e-4,
                                           d_frm.data_ptr(), d_cpl.data_ptr(), d_curr.data_ptr(), d_lc.data_ptr(),
                                           d_ld.data_ptr(), d_it.data_ptr(), d_err.data_ptr(), d_nc.data_ptr(),
                                           d_st.data_ptr(), ncs, nbl + 1, ctypes.c_void_p(s.cuda_stream))
        assert rc == 0
        s.synchronize()
        assert np.array_equal(d_curr.cpu().numpy()[:, :2], r["curr"])
        assert np.array_equal(d_lc.cpu().numpy()[:, :nbl - 1], r["layer_curr"])
        assert np.array_equal(d_ld.cpu().numpy()[:, :nbl], r["layer_dens"])
        assert np.array_equal(d_it.cpu().numpy(), r["scba_iter"])
        assert np.array_equal(d_st.cpu().numpy(), r["status"])
        # strides below the largest ncont / nbl are rejected
        rc = L.negf_b200_meir_wingreen_dev(gpu_ctx.handle, n, d_ids.data_ptr(), d_E.data_ptr(), 1e-4,
                                           d_frm.data_ptr(), d_cpl.data_ptr(), d_curr.data_ptr(), d_lc.data_ptr(),
                                           d_ld.data_ptr(), d_it.data_ptr(), d_err.data_ptr(), d_nc.data_ptr(),
                                           d_st.data_ptr(), 1, nbl, None)
        assert rc == native.BAD_ARG
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)


def test_elph_current_known_answer(gpu_ctx):
    """tests/f90elph_deph: zero coupling -> 2.0 +- 1e-4, coupling 0.05 -> [1.90, 1.95]"""
    dev = G.chain(10, 6, cblk=[6, 1])
    E = np.arange(-2.0, 2.0 + 1e-9, 0.1)
    did = gpu_ctx.upload(dev)
    gpu_ctx.set_options(scba_niter=5)
    try:
        r0 = gpu_ctx.meir_wingreen(did, E, [1.0, 0.0], coupling=np.zeros(60), eta=1e-4)
        c0 = O.integrate_el(r0["curr"][:, 0], -0.5, 0.5, 1e-3, 1e-3, -2.0, 2.0, 0.1) * 2
        r1 = gpu_ctx.meir_wingreen(did, E, [1.0, 0.0], coupling=np.full(60, 0.05), eta=1e-4)
        c1 = abs(O.integrate_el(r1["curr"][:, 0], -0.5, 0.5, 1e-3, 1e-3, -2.0, 2.0, 0.1) * 2)
        assert abs(c0 - 2.0) < 1e-4
        assert 1.90 <= c1 <= 1.95
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)


def test_ladder_known_answer(gpu_ctx):
    """Two orbitals per layer: a perfect ladder transmits one unit per open
    band (known answer, independent of the oracle)."""
    import sys
    import os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_oracle import _ladder
    dev = _ladder()
    E = np.array([-2.3, -1.8, -1.0, -0.2, 0.4, 1.2, 1.9, 2.2, 2.7])
    expect = np.array([sum(abs(e - s * 0.5) < 2.0 for s in (1, -1)) for e in E], dtype=float)
    did = gpu_ctx.upload(dev)
    try:
        T, nc, st = gpu_ctx.transmission(did, E, eta=1e-7)
        assert np.all(st == 0)
        assert np.abs(T - expect).max() < 1e-4
    finally:
        gpu_ctx.release(did)


@pytest.mark.parametrize("gen", ["c0", "c1_S"])
def test_bound_surface_parity(gpu_ctx, gen):
    """Contacts with bound surface layers (surfdim > 0, the bound-state block
    of surface_green, src/contselfenergy.F90:226-243): T and DOS against the
    oracle at the strict rule; periodic surface layers give the plain device's
    T; the mixed form declines them."""
    dev0 = (G.transport_c0(nbl=5, n=16, seed=4) if gen == "c0"
            else G.transport_c1(nbl=4, n=12, seed=4, density=0.3))
    dev = G.with_periodic_surface(G.with_periodic_surface(dev0, 0, 1), 1, 2)
    # an irregular surface too: perturb the surface-only entries so the answer is not the plain one
    rng = np.random.default_rng(3)
    n0 = dev.surf_size[0]
    bump = 0.05 * (rng.standard_normal((n0, n0)) + 1j * rng.standard_normal((n0, n0)))
    dev.lead_hs[0][:n0, :n0] += bump + bump.conj().T
    E = np.linspace(-1.8, 1.8, 13)
    did, d0 = gpu_ctx.upload(dev), gpu_ctx.upload(dev0)
    try:
        T, ncyc, st = gpu_ctx.transmission(did, E, eta=1e-6)
        ref, spread = oracle_spread(_o_T(E, eta=1e-6), dev, nsamp=2)
        assert np.all(st == ref["status"])
        assert np.array_equal(ncyc, ref["ncyc"])
        assert_T_strict(T, ref["T"], xp_reference(dev, E, 1e-6), spread=spread["T"], what="surface T")
        Td, dos, ncd, std = gpu_ctx.transmission_dos(did, E, eta=1e-6, dos_delta=1e-4)
        rd, sd = oracle_spread(_o_dos(E, eta=1e-6, dos_delta=1e-4), dev, nsamp=2)
        assert np.array_equal(ncd, rd["ncyc"])
        assert_parity(dos, rd["dos"], 1e-10 * max(np.abs(rd["dos"]).max(), 1.0), spread=sd["dos"], what="surface DOS",
                      rows=True)
        # periodic surface layers: the plain device's T
        per = gpu_ctx.upload(G.with_periodic_surface(dev0, 1, 1))
        try:
            Tp = gpu_ctx.transmission(per, E, eta=1e-4)[0]
            T0 = gpu_ctx.transmission(d0, E, eta=1e-4)[0]
            assert np.all(np.abs(Tp - T0) <= np.maximum(1e-10 * np.abs(T0), 1e-11))
        finally:
            gpu_ctx.release(per)
        gpu_ctx.set_options(precision=8)
        with pytest.raises(native.NegfError) as e:
            gpu_ctx.transmission(did, E, eta=1e-6)
        assert e.value.code == native.BAD_ARG
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)
        gpu_ctx.release(d0)


def test_c2_point_near_a_lead_resonance(gpu_ctx):
    """The block-512 device (60 layers, k = 0, S = I + 0.05 R) at grid point
    296 of 1024 on [-2, 2] eV, eta = 1e-6: the second contact's decimation is
    chaotic in FP64 (its Ao reaches condition 4e8 on the second iteration;
    under 1e-15 input perturbations the GPU iteration reached the retarded
    solution in 8 of 16 cases, the NumPy restatement diverged in 3 of 12,
    the LAPACK oracle stayed on it in 22 of 22).  A converged fixed point
    whose -Im gs has negative diagonal entries is detected and the
    decimation runs again from inputs a few ulps away: T matches the
    long-double value 2.22700 and the oracle within its FP64 scatter, through
    the engine and through the mixed form (which hands such a point to the
    engine)."""
    dev = G.transport_c1_kpoints([0.0], nbl=60, n=512, seed=1)[0]
    E = np.array([-0.8426197458455522])
    did = gpu_ctx.upload(dev)
    try:
        ref, spread = oracle_spread(_o_T(E, eta=1e-6), dev, nsamp=2)
        tol = max(10 * spread["T"][0], 2e-3)
        for opts in (dict(), dict(precision=8)):
            gpu_ctx.set_options(**opts)
            T, ncyc, st = gpu_ctx.transmission(did, E, eta=1e-6)
            assert np.all(st == 0), opts
            assert abs(T[0] - 2.22700145) <= tol, (opts, T, ref["T"], spread["T"])
            assert abs(T[0] - ref["T"][0]) <= tol, opts
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)
