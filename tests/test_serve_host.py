"""The request loop's host logic on CPU, with stand-in engine contexts: every
point of every request is solved once, batches mix requests of one solve
kind, later arrivals join running work, idle devices are evicted to admit new
ones, and an oversize device is rejected."""
import threading
import time

import numpy as np

from libnegf_b200 import generators as G
from libnegf_b200.serve import Request, Server


class FakeContext:
    """Records launches; T(E) = E * (device id + 1) per pair index + pair number."""

    def __init__(self):
        self.devices = {}
        self.next_id = 0
        self.launches = []
        self.released = []
        self.precision = 0
        self.shapes = []           # per launch: (precision option, {(block order, layers)} of its devices)
        self.lock = threading.Lock()

    def set_options(self, **kw): pass

    def update_options(self, **kw):
        self.precision = kw.get("precision", self.precision)

    def set_workspace_limit(self, n): pass
    def set_sgf_cache(self, mode, n=0): pass
    def set_tun_proj(self, did, p): pass
    def set_dos_proj(self, did, p): pass
    def close(self): pass

    def upload(self, dev):
        with self.lock:
            did = self.next_id
            self.next_id += 1
            self.devices[did] = dev
            return did

    def release(self, did):
        with self.lock:
            self.devices.pop(did)
            self.released.append(did)

    def transmissions(self, ids, E, pairs, eta=1e-4, ldos=False, dos_delta=1e-4, check=True):
        ids = np.asarray(ids)
        with self.lock:
            self.launches.append((tuple(sorted(set(ids.tolist()))), len(E), ldos))
            self.shapes.append((self.precision, {(max(self.devices[int(i)].pl_size), self.devices[int(i)].nbl)
                                                 for i in set(ids.tolist())}))
        time.sleep(0.01)
        T = np.stack([E * (ids + 1) + q for q in range(len(pairs))], axis=1)
        led = np.stack([E, -E], axis=1) if ldos else None
        return T, led, np.zeros(len(E), np.int32), np.zeros(len(E), np.int32)


def _expected(r, srv, lane=0):
    did = srv._resident[srv._key(r)].ids[lane] if srv._key(r) in srv._resident else None
    return did


def test_every_point_once_and_batches_mix_requests():
    ctxs = [FakeContext(), FakeContext()]
    srv = Server(contexts=ctxs, sms=4, points_per_launch=16, hbm_budget=1 << 34, sgf_cache_bytes=0)
    try:
        devs = [G.transport_c0(nbl=3, n=4, seed=s) for s in range(3)]
        reqs = [srv.submit(Request(devs[i], np.linspace(-1, 1, 10 + 7 * i), pairs=[(1, 2), (2, 1)])) for i in range(3)]
        time.sleep(0.02)
        late = srv.submit(Request(devs[0], np.linspace(0, 1, 9), pairs=[(1, 2), (2, 1)]))
        for r in reqs + [late]:
            assert r.wait(30) and r.error is None
        # device ids are the same in both lanes (uploaded in the same order)
        for r in reqs + [late]:
            did = srv._resident[srv._key(r)].ids[0]
            exp = np.stack([r.energies * (did + 1) + q for q in range(2)], axis=1)
            assert np.array_equal(r.T, exp)
        launches = ctxs[0].launches + ctxs[1].launches
        assert sum(n for _, n, _ in launches) == sum(r.energies.size for r in reqs + [late])
        assert all(n <= 16 for _, n, _ in launches)
        assert any(len(ids) > 1 for ids, _, _ in launches)          # points of several devices in one launch
        assert len(srv.latencies()) == 4
        assert srv.launches == len(launches)
    finally:
        srv.close()


def test_kinds_are_not_mixed_in_a_launch():
    ctxs = [FakeContext()]
    srv = Server(contexts=ctxs, sms=4, points_per_launch=64, hbm_budget=1 << 34, sgf_cache_bytes=0)
    try:
        d = G.transport_c0(nbl=3, n=4, seed=0)
        a = srv.submit(Request(d, np.linspace(-1, 1, 20)))
        b = srv.submit(Request(d, np.linspace(-1, 1, 20), ldos=True, dos_proj=[[1], [2]]))
        assert a.wait(30) and b.wait(30)
        assert a.ledos is None and b.ledos.shape == (20, 2)
        assert np.array_equal(b.ledos[:, 0], b.energies)
        kinds = {(n, l) for _, n, l in ctxs[0].launches}
        assert all(isinstance(l, bool) for _, l in kinds)
    finally:
        srv.close()


def test_eviction_and_rejection():
    ctxs = [FakeContext()]
    one = G.transport_c0(nbl=3, n=4, seed=0)
    budget_dev = one.nbytes() + 100                     # room for one such device at a time
    srv = Server(contexts=ctxs, sms=4, points_per_launch=8, hbm_budget=budget_dev * 3, sgf_cache_bytes=0)
    srv.dev_budget = budget_dev                          # pin the device share for the test
    try:
        r1 = srv.submit(Request(one, np.linspace(-1, 1, 8)))
        assert r1.wait(30) and r1.error is None
        other = G.transport_c0(nbl=3, n=4, seed=1)
        r2 = srv.submit(Request(other, np.linspace(-1, 1, 8)))
        assert r2.wait(30) and r2.error is None
        assert ctxs[0].released == [0]                   # the idle first device made room
        big = G.transport_c0(nbl=12, n=8, seed=2)
        r3 = srv.submit(Request(big, np.linspace(-1, 1, 4)))
        assert r3.wait(30) and r3.error is not None and np.all(r3.status == 8)
    finally:
        srv.close()


def test_srpt_takes_the_least_remaining_work_first():
    """The batch order: "srpt" starts with the request whose pending points
    cost least in total, "fifo" with the oldest points; results are not
    affected either way (every point is solved once, as above)."""
    big_dev = G.transport_c0(nbl=6, n=8, seed=0)
    small_dev = G.transport_c0(nbl=3, n=4, seed=1)
    for policy, first in (("srpt", "small"), ("fifo", "big")):
        srv = Server(contexts=[FakeContext()], sms=4, points_per_launch=16, hbm_budget=1 << 34, sgf_cache_bytes=0,
                     policy=policy)
        srv.close()                                   # drive _take_batch by hand
        big = Request(big_dev, np.linspace(-1, 1, 100))
        small = Request(small_dev, np.linspace(-1, 1, 5))
        srv._pending = [(big, i) for i in range(100)] + [(small, i) for i in range(5)]
        batch = srv._take_batch()
        assert len(srv._pending) == 105 - len(batch)
        if first == "small":
            # the big request's points cost more than 4x the small one's: not in this batch
            assert len(batch) == 5 and all(r is small for r, _ in batch)
        else:
            assert len(batch) == 16 and all(r is big for r, _ in batch) and [i for _, i in batch] == list(range(16))


def test_out_of_order_completion():
    """With "srpt" a small request that arrives after a large one finishes
    first; the loop's bookkeeping of active requests must not compare
    requests by value (they hold arrays)."""
    ctxs = [FakeContext()]
    srv = Server(contexts=ctxs, sms=4, points_per_launch=16, hbm_budget=1 << 34, sgf_cache_bytes=0, policy="srpt")
    try:
        big = srv.submit(Request(G.transport_c0(nbl=4, n=8, seed=0), np.linspace(-1, 1, 200)))
        time.sleep(0.005)
        small = srv.submit(Request(G.transport_c0(nbl=3, n=4, seed=1), np.linspace(-1, 1, 5)))
        assert small.wait(30) and big.wait(30)
        assert small.error is None and big.error is None
        assert small.t_done < big.t_done
    finally:
        srv.close()


def test_mixed_precision_requests_batch_by_precision_and_shape():
    """Mixed-form requests share a launch only with requests of the same
    precision, block order and layer count (the lock-step call needs one
    shape); the lane sets its precision option per batch; FP64 requests of any
    shape still mix.  A mixed request the form cannot take (LDOS) fails at
    submission with BAD_ARG."""
    from libnegf_b200 import native
    ctxs = [FakeContext(), FakeContext()]
    srv = Server(contexts=ctxs, sms=4, points_per_launch=16, hbm_budget=1 << 34, sgf_cache_bytes=0)
    reqs = []
    for q, (n, nbl, prec) in enumerate([(8, 4, 8), (8, 4, 8), (16, 4, 8), (8, 5, 7), (8, 4, 0), (16, 5, 0),
                                        (8, 4, 1)]):
        dev = G.transport_c0(nbl=nbl, n=n, seed=q)
        reqs.append(srv.submit(Request(dev, np.linspace(-1, 1, 20 + q), precision=prec)))
    bad = srv.submit(Request(G.transport_c0(nbl=4, n=8, seed=9), np.linspace(-1, 1, 5), precision=8, ldos=True,
                             dos_proj=[[1, 2]]))
    assert bad.wait(1) and bad.error and np.all(bad.status == native.BAD_ARG)
    for r in reqs:
        assert r.wait(30) and r.error is None
    srv.close()
    for r in reqs:                                     # every point solved once, in its own request
        did = srv._resident[srv._key(r)].ids[0]
        assert np.array_equal(r.T[:, 0], r.energies * (did + 1)) and not r.status.any()
    shapes = [sh for c in ctxs for sh in c.shapes]
    assert sum(len(c.launches) for c in ctxs) == srv.launches
    for prec, devs in shapes:
        if prec:
            assert len(devs) == 1, devs                # one shape per mixed launch
    precs = {p for p, _ in shapes}
    assert {0, 1, 7, 8} <= precs
