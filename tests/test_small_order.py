"""The lock-step schedule of 2-contact transmission solves at small orders
(options.schedule; n <= 32): every point of a call through the same block
operation at once, one warp per point and operation, complex FP64.  Held to
the same strict parity as the persistent engine (1e-10 relative / 1e-13
absolute, decimation iteration counts equal to the oracle's, points listed
only where the CPU FP64 paths themselves scatter), and to the engine's
status rules."""
import ctypes

import numpy as np
import pytest

from conftest import assert_T_strict, oracle_spread, xp_reference
from golden.make_config_shapes import CASES as SHAPES, PATH, fingerprint
from libnegf_b200 import generators as G
from libnegf_b200 import native
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SMALL = {
    "chain_n1": lambda: (G.chain(1, 4), np.linspace(-1.9, 1.9, 9)),
    "chain3_rev": lambda: (G.chain(3, 5, cblk=[5, 1]), np.linspace(-1.9, 1.9, 9)),
    "c0_n5": lambda: (G.transport_c0(nbl=7, n=5, seed=2), np.linspace(-3, 3, 33)),
    "c1_S_n16": lambda: (G.transport_c1(nbl=6, n=16, seed=2, density=0.3), np.linspace(-2, 2, 33)),
    "c0_n17": lambda: (G.transport_c0(nbl=5, n=17, seed=3), np.linspace(-3, 3, 33)),
    "c1_S_n32": lambda: (G.transport_c1(nbl=8, n=32, seed=4, density=0.2), np.linspace(-2, 2, 33)),
}


def _T(ctx, did, E, eta, schedule, **opt):
    ctx.set_options(schedule=schedule, **opt)
    try:
        return ctx.transmission(did, E, eta=eta, check=False)
    finally:
        ctx.set_options()


@pytest.mark.parametrize("case", sorted(SMALL))
def test_lockstep_parity(gpu_ctx, case):
    dev, E = SMALL[case]()
    did = gpu_ctx.upload(dev)
    try:
        T, ncyc, st = _T(gpu_ctx, did, E, 1e-6, 2)
        ref, spread = oracle_spread(lambda d: dict(zip(("T", "ncyc", "status"), O.transmission(d, E, eta=1e-6))),
                                    dev, nsamp=2)
        assert np.all(st == ref["status"])
        assert np.array_equal(ncyc, ref["ncyc"])
        assert_T_strict(T, ref["T"], xp_reference(dev, E, 1e-6), spread=spread["T"], what=case)
    finally:
        gpu_ctx.release(did)


@pytest.mark.parametrize("schedule", [1, 2])
def test_c0_shape_both_schedules(gpu_ctx, schedule):
    """The CPU-runnable config (N = 20, n = 32, all 512 energies, SGFACC =
    1e-12) through the engine and through lock step, against the fixture."""
    z = np.load(PATH)
    devs, ids, E, p = SHAPES["c0"]()
    assert fingerprint(devs[0]) == str(z["c0__fp0"])
    E = np.array(z["c0__E"])
    did = gpu_ctx.upload(devs[0])
    try:
        T, ncyc, st = _T(gpu_ctx, did, E, p["eta"], schedule, sgf_tol=p["sgf_tol"])
        assert np.all(st == 0)
        assert np.array_equal(ncyc, z["c0__ncyc_o"])
        x = {"T_x": z["c0__T_x"], "T_d": z["c0__T_d"], "T_g": z["c0__T_g"]}
        assert_T_strict(T, z["c0__T_o"], x, spread=z["c0__T_s"], what="c0 schedule %d" % schedule)
    finally:
        gpu_ctx.release(did)


def test_lockstep_point_is_independent_of_its_batch(gpu_ctx):
    """A point's result does not depend on the other points of the call, their
    order, or how the call is cut into batches by the workspace limit."""
    devs = G.transport_c1_kpoints([0.0, 1.1], nbl=6, n=24, seed=9, density=0.2)
    hs = [gpu_ctx.upload(d) for d in devs]
    try:
        E = np.linspace(-2, 2, 40)
        ids = np.repeat(np.asarray(hs, dtype=np.int32), E.size)
        EE = np.tile(E, len(hs))
        T0, n0, s0 = _T(gpu_ctx, ids, EE, 1e-6, 2)
        perm = np.random.default_rng(3).permutation(EE.size)
        T1, n1, s1 = _T(gpu_ctx, ids[perm], EE[perm], 1e-6, 2)
        assert np.array_equal(T1, T0[perm]) and np.array_equal(n1, n0[perm])
        sub = perm[:7]
        T2, n2, _ = _T(gpu_ctx, ids[sub], EE[sub], 1e-6, 2)
        assert np.array_equal(T2, T0[sub])
        gpu_ctx.set_workspace_limit(3 * 13 * 24 * 24 * 16 + 4096)    # a few points per batch
        try:
            T3, n3, _ = _T(gpu_ctx, ids, EE, 1e-6, 2)
        finally:
            gpu_ctx.set_workspace_limit(0)
        assert np.array_equal(T3, T0) and np.array_equal(n3, n0)
        # the auto schedule takes lock step for these points: the same bits
        T4, _, _ = _T(gpu_ctx, ids, EE, 1e-6, 0)
        assert np.array_equal(T4, T0)
    finally:
        for h in hs:
            gpu_ctx.release(h)


def test_schedule_rules(gpu_ctx):
    """schedule 2 refuses what lock step does not cover; auto (0) hands it to
    the engine, bit for bit what schedule 1 gives."""
    E = np.linspace(-1, 1, 5)
    cases = [G.transport_c0(nbl=4, n=33, seed=1),                      # n > 32
             G.transport_c0(nbl=6, n=8, seed=1, cblk=[2, 5]),          # contacts off blocks 1 and nbl
             G.uneven([5, 7, 3, 6], seed=4)]                           # uneven PLs
    hs = [gpu_ctx.upload(d) for d in cases]
    try:
        for h in hs:
            with pytest.raises(native.NegfError) as e:
                _T(gpu_ctx, h, E, 1e-6, 2)
            assert e.value.code == native.BAD_ARG
            Ta, na, sa = _T(gpu_ctx, h, E, 1e-6, 0)
            Tb, nb, sb = _T(gpu_ctx, h, E, 1e-6, 1)
            assert np.array_equal(Ta, Tb) and np.array_equal(na, nb) and np.array_equal(sa, sb)
        ok = gpu_ctx.upload(G.transport_c0(nbl=3, n=8, seed=2))
        hs.append(ok)
        gpu_ctx.set_options(schedule=2)
        try:
            with pytest.raises(native.NegfError) as e:             # DOS is the engine's
                gpu_ctx.transmission_dos(ok, E, eta=1e-6)
            assert e.value.code == native.BAD_ARG
        finally:
            gpu_ctx.set_options()
        with pytest.raises(native.NegfError) as e:
            gpu_ctx.set_options(schedule=3)
        assert e.value.code == native.BAD_ARG
    finally:
        for h in hs:
            gpu_ctx.release(h)


def test_lockstep_dev_call_matches_host_call(gpu_ctx):
    torch = pytest.importorskip("torch")
    dev = G.transport_c1(nbl=6, n=20, seed=5, density=0.25)
    E = np.linspace(-2, 2, 50)
    did = gpu_ctx.upload(dev)
    L = native.load()
    try:
        Th, nh, sh = _T(gpu_ctx, did, E, 1e-6, 2)
        n = E.size
        d_ids = torch.full((n,), did, dtype=torch.int32, device="cuda")
        d_E = torch.from_numpy(E).cuda()
        d_T = torch.zeros(n, dtype=torch.float64, device="cuda")
        d_nc = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_st = torch.zeros(n, dtype=torch.int32, device="cuda")
        s = torch.cuda.Stream()
        gpu_ctx.set_options(schedule=0)
        rc = L.negf_b200_transmission_dev(gpu_ctx.handle, n, d_ids.data_ptr(), d_E.data_ptr(), 1e-6, 1, 2,
                                          d_T.data_ptr(), d_nc.data_ptr(), d_st.data_ptr(),
                                          ctypes.c_void_p(s.cuda_stream))
        s.synchronize()
        assert rc == 0
        assert np.array_equal(d_T.cpu().numpy(), Th)
        assert np.array_equal(d_nc.cpu().numpy(), nh)
        # under stream capture the auto schedule hands the call to the engine
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            rc = L.negf_b200_transmission_dev(gpu_ctx.handle, n, d_ids.data_ptr(), d_E.data_ptr(), 1e-6, 1, 2,
                                              d_T.data_ptr(), d_nc.data_ptr(), d_st.data_ptr(),
                                              ctypes.c_void_p(s.cuda_stream))
        assert rc == 0
        g.replay()
        torch.cuda.synchronize()
        Te, ne, _ = _T(gpu_ctx, did, E, 1e-6, 1)
        assert np.array_equal(d_T.cpu().numpy(), Te)
        del g
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)


def test_lockstep_statuses_match_the_engine(gpu_ctx):
    """An iteration cap below what the decimation needs: NOT_CONVERGED and
    ncyc = cap + 1 on the same points as the engine; a NaN planted in H: a
    non-zero status on every point, and the context stays usable."""
    dev = G.transport_c0(nbl=5, n=16, seed=6)
    E = np.linspace(-2.5, 2.5, 21)
    did = gpu_ctx.upload(dev)
    bad = G.transport_c0(nbl=5, n=16, seed=6)
    bad.h_diag[3][2, 9] = np.nan
    bid = gpu_ctx.upload(bad)
    try:
        Tl, nl, sl = _T(gpu_ctx, did, E, 1e-6, 2, sgf_max_iter=6)
        Te, ne, se = _T(gpu_ctx, did, E, 1e-6, 1, sgf_max_iter=6)
        assert np.array_equal(sl, se) and np.array_equal(nl, ne)
        assert np.any(sl == native.NOT_CONVERGED)
        Tb, nb, sb = _T(gpu_ctx, bid, E, 1e-6, 2)
        assert np.all(sb != 0)
        T, ncyc, st = _T(gpu_ctx, did, E, 1e-6, 2)
        assert np.all(st == 0)
        Tr, ncr, _ = O.transmission(dev, E, eta=1e-6)
        assert np.array_equal(ncyc, ncr)
    finally:
        gpu_ctx.release(did)
        gpu_ctx.release(bid)
