"""Serving: the surface Green's function cache, the workspace cap and the
continuous-batching request loop (results the same alone and in the mix)."""
import time

import numpy as np
import pytest

from conftest import assert_parity, assert_T_close, oracle_spread
from libnegf_b200 import generators as G
from oracle import oracle as O


@pytest.mark.gpu
def test_sgf_cache_reuses_surface_gf(gpu_ctx):
    """The cache lives in the persistent engine: the uncached reference call
    runs there too (schedule 1), so the bits compare."""
    dev = G.transport_c0(nbl=6, n=8, seed=0)
    E = np.linspace(-2.5, 2.5, 21)
    did = gpu_ctx.upload(dev)
    gpu_ctx.set_options(schedule=1)
    try:
        T0, nc0, st0 = gpu_ctx.transmission(did, E, eta=1e-6)
        gpu_ctx.set_sgf_cache(1, 64 << 20)
        T1, nc1, _ = gpu_ctx.transmission(did, E, eta=1e-6)      # fills the cache
        s1 = gpu_ctx.sgf_cache_stats()
        T2, nc2, _ = gpu_ctx.transmission(did, E, eta=1e-6)      # all hits
        s2 = gpu_ctx.sgf_cache_stats()
        assert s1["entries"] == 2 * E.size and s2["hits"] - s1["hits"] == 2 * E.size
        assert np.array_equal(T0, T1) and np.array_equal(T1, T2)
        assert np.array_equal(nc1, nc0) and np.all(nc2 == 0)     # loaded: no decimation (reference: ncyc = 0)
        # the DOS solve at the same E + i*eta reuses them too
        Td, dos, ncd, _ = gpu_ctx.transmission_dos(did, E, eta=1e-6, dos_delta=1e-4)
        assert np.all(ncd == 0)
        ref = O.transmission_dos(dev, E, eta=1e-6, dos_delta=1e-4)
        assert_T_close(Td, ref[0], rtol=1e-9)
        # another eta is another label
        _, nc3, _ = gpu_ctx.transmission(did, E, eta=1e-5)
        assert np.all(nc3 > 0)
        # refresh mode recomputes
        gpu_ctx.set_sgf_cache(2, 64 << 20)
        T4, nc4, _ = gpu_ctx.transmission(did, E, eta=1e-6)
        assert np.all(nc4 > 0) and np.array_equal(T4, T0)
    finally:
        gpu_ctx.set_options()
        gpu_ctx.set_sgf_cache(0)
        gpu_ctx.release(did)


@pytest.mark.gpu
def test_sgf_cache_file_round_trip(tmp_path):
    """Saved surface GFs are read back in another context (other device ids)
    and by a device that only shares the leads: all hits, the same T."""
    import copy
    from libnegf_b200 import native
    dev = G.transport_c0(nbl=5, n=16, seed=2)
    other = copy.deepcopy(dev)
    other.h_diag[2] = other.h_diag[2] + 0.1 * np.eye(16)        # same leads, another interior
    E = np.linspace(-2.5, 2.5, 13)
    path = str(tmp_path / "sgf.bin")
    with native.Context(0) as c1:
        c1.set_sgf_cache(1, 64 << 20)
        d1 = c1.upload(dev)
        T1, nc1, _ = c1.transmission(d1, E, eta=1e-6)
        assert c1.sgf_cache_save(path) == 2 * E.size
    with native.Context(0) as c2:
        c2.set_sgf_cache(1, 64 << 20)
        c2.upload(G.transport_c0(nbl=3, n=8, seed=9))              # shifts the device ids
        d2 = c2.upload(dev)
        d3 = c2.upload(other)
        assert c2.sgf_cache_load(path) == 2 * E.size
        s0 = c2.sgf_cache_stats()
        T2, nc2, _ = c2.transmission(d2, E, eta=1e-6)
        T3, nc3, _ = c2.transmission(d3, E, eta=1e-6)
        s1 = c2.sgf_cache_stats()
        assert s1["hits"] - s0["hits"] == 4 * E.size and s1["misses"] == s0["misses"]
        assert np.array_equal(T2, T1) and np.all(nc2 == 0) and np.all(nc3 == 0)
        ref, spread = oracle_spread(lambda d: O.transmission(d, E, eta=1e-6)[0], other)
        assert_T_close(T3, ref, spread=spread)
        # another broadening is not in the file
        _, nc4, _ = c2.transmission(d2, E, eta=1e-5)
        assert np.all(nc4 > 0)


@pytest.mark.gpu
def test_workspace_limit_runs_fewer_ctas(gpu_ctx):
    from libnegf_b200 import native
    dev = G.transport_c0(nbl=8, n=32, seed=3)
    E = np.linspace(-2, 2, 64)
    did = gpu_ctx.upload(dev)
    gpu_ctx.set_options(schedule=1)                               # the persistent engine's CTAs
    try:
        T0, _, _ = gpu_ctx.transmission(did, E, eta=1e-6)
        slot = 32 * 32 * 16
        gpu_ctx.set_workspace_limit(256 + 3 * 40 * slot)         # about three CTAs
        T1, _, _ = gpu_ctx.transmission(did, E, eta=1e-6)
        assert np.array_equal(T0, T1)
        gpu_ctx.set_workspace_limit(1024)                         # not one CTA
        with pytest.raises(native.NegfError) as ei:
            gpu_ctx.transmission(did, E, eta=1e-6)
        assert ei.value.code == native.ADMISSION
    finally:
        gpu_ctx.set_options()
        gpu_ctx.set_workspace_limit(0)
        gpu_ctx.release(did)


def _requests():
    from libnegf_b200.serve import Request
    a = Request(G.transport_c0(nbl=12, n=16, seed=1), np.linspace(-2.8, 2.8, 97), eta=1e-6)
    b = Request(G.transport_c0(nbl=6, n=64, seed=2), np.linspace(-2, 2, 41), eta=1e-6, pairs=[(2, 1)])
    c = Request(G.transport_c0(nbl=5, n=32, seed=3, cblk=[1, 5, 3]), np.linspace(-2, 2, 33), eta=1e-6,
                pairs=[(1, 2), (1, 3)], ldos=True, dos_delta=1e-4, dos_proj=[[1, 2, 3], list(range(33, 65))])
    d = Request(G.uneven([5, 9, 4, 7], seed=4), np.linspace(-2, 2, 29), eta=1e-4)
    return [a, b, c, d]


@pytest.mark.gpu
def test_same_alone_and_in_the_mix():
    """Each request alone on the server, then all of them with staggered
    arrivals (later ones join while earlier launches run): identical
    results, and each matches the oracle."""
    from libnegf_b200.serve import Server
    alone = {}
    srv = Server(lanes=2, points_per_launch=24, hbm_budget=8 << 30, sgf_cache_bytes=64 << 20)
    try:
        for i, r in enumerate(_requests()):
            srv.submit(r)
            assert r.wait(120)
            assert r.error is None
            alone[i] = (r.T.copy(), None if r.ledos is None else r.ledos.copy())
    finally:
        srv.close()
    srv = Server(lanes=2, points_per_launch=24, hbm_budget=8 << 30, sgf_cache_bytes=64 << 20)
    try:
        reqs = _requests()
        for r in reqs[:2]:
            srv.submit(r)
        time.sleep(0.05)
        for r in reqs[2:]:
            srv.submit(r)
        for r in reqs:
            assert r.wait(120)
        for i, r in enumerate(reqs):
            assert r.error is None and np.all(r.status == 0)
            assert np.array_equal(r.T, alone[i][0])
            if r.ldos:
                assert np.array_equal(r.ledos, alone[i][1])
            kw = dict(eta=r.eta, dos_proj=r.dos_proj, dos_delta=r.dos_delta) if r.ldos else dict(eta=r.eta)
            ref, spread = oracle_spread(lambda d: O.transmissions(d, r.energies, r.pairs, **kw)[0], r.device)
            assert_T_close(r.T, ref, spread=spread)
        lat = srv.latencies()
        assert lat.size == 4 and np.all(lat > 0)
    finally:
        srv.close()


@pytest.mark.gpu
def test_admission_rejects_a_device_over_budget():
    from libnegf_b200 import native
    from libnegf_b200.serve import Request, Server
    srv = Server(lanes=1, hbm_budget=64 << 20, sgf_cache_bytes=1 << 20)
    try:
        big = Request(G.transport_c0(nbl=100, n=128, seed=5), np.linspace(-1, 1, 4))   # ~80 MB of blocks
        small = Request(G.transport_c0(nbl=4, n=8, seed=6), np.linspace(-1, 1, 4))
        srv.submit(big)
        srv.submit(small)
        assert big.wait(60) and small.wait(60)
        assert big.error is not None and np.all(big.status == native.ADMISSION)
        assert small.error is None and np.all(small.status == 0)
    finally:
        srv.close()


@pytest.mark.gpu
def test_mixed_precision_requests_in_the_mix():
    """Mixed-form requests (8 int8 digits) served beside FP64 requests, on
    lanes that keep an SGF cache: each is bitwise the direct mixed-form call
    on the same points (whatever the batch cut) and within the mixed form's
    bound, max(1e-8 |T|, 1e-11), of the oracle; the FP64 requests beside them
    keep their alone results."""
    from libnegf_b200 import native
    from libnegf_b200.serve import Request, Server
    devs = [G.transport_c0(nbl=4, n=128, seed=21), G.transport_c0(nbl=5, n=16, seed=22)]
    Es = [np.linspace(-2.0, 2.0, 20), np.linspace(-2.5, 2.5, 40)]
    direct = []
    with native.Context(0) as ctx:
        ctx.set_options(precision=8)
        for dev, E in zip(devs, Es):
            did = ctx.upload(dev)
            direct.append(ctx.transmission(did, E, eta=1e-4, check=False))
            ctx.release(did)
    alone = []
    srv = Server(lanes=2, points_per_launch=24, hbm_budget=8 << 30, sgf_cache_bytes=64 << 20)
    try:
        for r in _requests()[:2]:
            srv.submit(r)
            assert r.wait(120) and r.error is None
            alone.append(r.T.copy())
    finally:
        srv.close()
    srv = Server(lanes=2, points_per_launch=24, hbm_budget=8 << 30, sgf_cache_bytes=64 << 20)
    try:
        mixed = [Request(d, E, eta=1e-4, precision=8) for d, E in zip(devs, Es)]
        plain = _requests()[:2]
        for r in plain[:1] + mixed + plain[1:]:
            srv.submit(r)
        for r in mixed + plain:
            assert r.wait(120) and r.error is None and np.all(r.status == 0)
        for r, T0 in zip(plain, alone):
            assert np.array_equal(r.T, T0)
        for r, (T, nc, st) in zip(mixed, direct):
            assert not st.any()
            assert np.array_equal(r.T[:, 0], T) and np.array_equal(r.ncyc, nc)
            ref, spread = oracle_spread(lambda d: O.transmission(d, r.energies, eta=1e-4)[0], r.device, nsamp=2)
            assert_parity(r.T[:, 0], ref, np.maximum(1e-8 * np.abs(ref), 1e-11), spread=spread, what="served mixed T")
    finally:
        srv.close()
