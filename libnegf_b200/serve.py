"""Request loop for transmission / DOS solves with continuous batching.

Requests (a device, an energy grid, contact pairs, optional projections)
arrive at any time from any thread.  The loop keeps every device of an
admitted request resident in HBM (H/S and contact blocks uploaded once per
lane, with its projections), keeps the contact surface Green's functions of
solved points in each lane's device cache (the ln_cache counterpart), and
feeds the GPU from a pool of pending energy points:

- lanes: independent engine contexts on the same GPU, each with its own
  stream and workspace; a lane runs one persistent launch at a time, and
  the launches of different lanes run concurrently on the SMs;
- batching: whenever a lane is free it takes pending points of one solve
  kind (T or T+LDOS, same eta, dos_delta, pairs and precision; for the mixed
  form also the same block order and layer count, since its lock-step call
  needs one shape), whatever request they belong to, up to
  `points_per_launch`, and sets its `precision` option for the batch;
  points of requests that arrived while other launches were running join
  the next launch of any free lane (continuous batching, not a queue of
  whole requests).  The order is
  `policy`: "fifo" (default) takes the oldest points first; "srpt" takes
  first the points of the request with the least estimated remaining work
  (pending points x a per-point cost of (layers + 80) x block order^3, the
  sweep plus the two leads' decimation), and fills the batch only with
  points at most 4x as costly as its first one; no result changes.  On the
  streams measured (B200, 2 lanes) srpt did not lower the latencies:
  launches are not preempted, and waiting behind a running batch of large
  points dominates;
- admission: a request is admitted when its device fits the HBM budget next
  to the resident devices (idle devices are evicted, least recently used
  first); a device larger than the budget on its own is rejected with
  NEGF_B200_ERR_ADMISSION.  The engine workspace of each lane is capped at
  its share of the budget, so a large block size runs on fewer CTAs instead
  of failing.

Per point the engine computes exactly the same thing whichever batch or lane
it lands in, so a request's results are the same alone and in the mix.
Latency of a request = completion of its last point - submission.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import native
from .device import Device


@dataclass(eq=False)   # identity: requests hold arrays, and two requests are never "equal"
class Request:
    device: Device
    energies: np.ndarray
    pairs: Sequence[Tuple[int, int]] = ((1, 2),)
    eta: float = 1e-4
    ldos: bool = False
    dos_delta: float = 1e-4
    tun_proj: Optional[Sequence[int]] = None
    dos_proj: Optional[Sequence[Sequence[int]]] = None
    key: Optional[object] = None          # device identity for reuse across requests (default: the object)
    # 0: complex FP64; 1 or 4..8: the mixed form (int8 tensor-core products with
    # that many digits, 1 = 8), for single-pair T requests (no LDOS, no tun_proj)
    # on devices with 2 contacts on blocks 1 and nbl and one PL size
    precision: int = 0
    # filled by the server
    T: Optional[np.ndarray] = None
    ledos: Optional[np.ndarray] = None
    ncyc: Optional[np.ndarray] = None
    status: Optional[np.ndarray] = None
    error: Optional[str] = None
    t_submit: float = 0.0
    t_done: float = 0.0
    _left: int = 0
    _done: threading.Event = field(default_factory=threading.Event)

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit

    def wait(self, timeout: Optional[float] = None) -> bool:
        return self._done.wait(timeout)


@dataclass(eq=False)
class _Resident:
    ids: List[int]                        # device id in every lane
    nbytes: int
    device: object = None                 # held, so that an id()-based key is never reused while resident
    users: int = 0
    last_use: float = 0.0


class Server:
    """Continuous-batching request loop on one GPU (see the module docstring)."""

    def __init__(self, cuda_device: int = 0, lanes: int = 2, points_per_launch: int = 0,
                 hbm_budget: int = 0, sgf_cache_bytes: int = 1 << 30, options: Optional[dict] = None,
                 contexts: Optional[list] = None, sms: int = 0, policy: str = "fifo"):
        """`contexts` (one per lane) and `sms` replace the engine contexts and
        the device query, for driving the loop with stand-ins.  `policy`:
        "srpt" or "fifo" (see the module docstring)."""
        if policy not in ("srpt", "fifo"):
            raise ValueError("policy must be 'srpt' or 'fifo'")
        self.policy = policy
        if contexts is not None:
            self.lanes = list(contexts)
            lanes = len(self.lanes)
        else:
            self.lanes = [native.Context(cuda_device) for _ in range(lanes)]
        if not sms or not hbm_budget:
            import torch
            if not sms:
                sms = torch.cuda.get_device_properties(cuda_device).multi_processor_count
            if not hbm_budget:
                free, _ = torch.cuda.mem_get_info(cuda_device)
                hbm_budget = int(free * 0.8)
        self.sms = sms
        self.budget = hbm_budget
        # the budget is split: resident devices, then per-lane workspace + cache
        self.ws_share = int(self.budget * 0.6) // lanes
        self.dev_budget = self.budget - self.ws_share * lanes - sgf_cache_bytes * lanes
        if self.dev_budget <= 0:
            raise ValueError("HBM budget too small for the workspace and cache shares")
        for ctx in self.lanes:
            if options:
                ctx.set_options(**options)
            ctx.set_workspace_limit(self.ws_share)
            if sgf_cache_bytes:
                ctx.set_sgf_cache(1, sgf_cache_bytes)
        # points per launch: enough to keep one lane's CTAs busy twice over
        self.ppl = points_per_launch or 2 * self.sms
        self._lock = threading.Lock()
        self._cv = threading.Condition(self._lock)
        self._arrivals: List[Request] = []
        self._active: List[Request] = []
        self._pending: List[Tuple[Request, int]] = []   # (request, point index)
        self._resident: Dict[object, _Resident] = {}
        self._stop = False
        self._threads = [threading.Thread(target=self._lane_loop, args=(i,), daemon=True) for i in range(lanes)]
        self._sched = threading.Thread(target=self._admit_loop, daemon=True)
        self.completed: List[Request] = []
        self.points_done = 0
        self.launches = 0          # engine launches (one per lane batch)
        self._sched.start()
        for t in self._threads:
            t.start()

    # ---------------------------------------------------------------- API
    def submit(self, req: Request) -> Request:
        req.energies = np.ascontiguousarray(req.energies, dtype=np.float64).ravel()
        req.t_submit = time.perf_counter()
        npts, npairs = req.energies.size, len(req.pairs)
        req.T = np.zeros((npts, npairs))
        req.ncyc = np.zeros(npts, dtype=np.int32)
        req.status = np.zeros(npts, dtype=np.int32)
        req._left = npts
        with self._cv:
            why = self._mixed_refusal(req)
            if why:                                   # the mixed form cannot take it: fails at once
                req.error = why
                req.status[:] = native.BAD_ARG
                self._finish(req)
                return req
            self._arrivals.append(req)
            self._cv.notify_all()
        return req

    @staticmethod
    def _mixed_refusal(req) -> Optional[str]:
        p = int(req.precision)
        if p == 0:
            return None
        if p != 1 and not 4 <= p <= 8:
            return "precision must be 0, 1 or 4..8"
        if req.ldos or len(req.pairs) != 1 or req.tun_proj is not None:
            return "the mixed form serves single-pair T requests without LDOS or tun_proj"
        return None

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads + [self._sched]:
            t.join(timeout=60)
        for ctx in self.lanes:
            ctx.close()

    def latencies(self) -> np.ndarray:
        return np.array([r.latency for r in self.completed if r.error is None])

    # ---------------------------------------------------------------- admission
    def _key(self, req):
        return req.key if req.key is not None else id(req.device)

    def _admit_one(self, req) -> bool:
        """Makes req's device resident in every lane; False if it must wait."""
        k = self._key(req)
        r = self._resident.get(k)
        if r is None:
            nbytes = req.device.nbytes() * len(self.lanes)
            if nbytes > self.dev_budget:
                req.error = "device of %d bytes exceeds the HBM budget of %d" % (nbytes, self.dev_budget)
                req.status[:] = native.ADMISSION
                self._finish(req)
                return True
            used = sum(x.nbytes for x in self._resident.values())
            # evict idle devices, least recently used first
            for kk, rr in sorted(self._resident.items(), key=lambda kv: kv[1].last_use):
                if used + nbytes <= self.dev_budget:
                    break
                if rr.users == 0:
                    for ctx, did in zip(self.lanes, rr.ids):
                        ctx.release(did)
                    used -= rr.nbytes
                    del self._resident[kk]
            if used + nbytes > self.dev_budget:
                return False
            ids = []
            for ctx in self.lanes:
                did = ctx.upload(req.device)
                ctx.set_tun_proj(did, req.tun_proj)
                ctx.set_dos_proj(did, req.dos_proj)
                ids.append(did)
            r = _Resident(ids=ids, nbytes=nbytes, device=req.device)
            self._resident[k] = r
        r.users += 1
        r.last_use = time.perf_counter()
        self._active.append(req)
        self._pending.extend((req, i) for i in range(req.energies.size))
        return True

    def _admit_loop(self):
        with self._cv:
            while not self._stop:
                waiting = []
                for req in self._arrivals:
                    if not self._admit_one(req):
                        waiting.append(req)
                self._arrivals = waiting
                self._cv.notify_all()
                self._cv.wait(timeout=0.05)

    # ---------------------------------------------------------------- batching
    @staticmethod
    def _group(req):
        p = int(req.precision)
        shape = (max(req.device.pl_size), int(req.device.nbl)) if p else None
        return (bool(req.ldos), float(req.eta), float(req.dos_delta) if req.ldos else 0.0, tuple(req.pairs), p, shape)

    @staticmethod
    def _point_cost(req) -> float:
        """Relative cost of one point: the sweep over the layers plus the two
        leads' decimation (about 40 iterations of a few products each)."""
        n = max(req.device.pl_size)
        return (req.device.nbl + 80.0) * float(n) ** 3

    def _take_batch(self):
        """Pending points of one solve kind, across requests, in policy order."""
        if not self._pending:
            return None
        if self.policy == "fifo":
            order = self._pending
        else:
            left = {}
            for r, _ in self._pending:
                left[id(r)] = left.get(id(r), 0) + 1
            # stable: within a request and among equal work, arrival order is kept
            order = sorted(self._pending, key=lambda it: left[id(it[0])] * self._point_cost(it[0]))
        g = self._group(order[0][0])
        # srpt: a batch ends when its slowest point does, so it takes only points
        # at most 4x as costly as the first one's (cheap requests do not wait on
        # expensive points launched beside them)
        cap = 4.0 * self._point_cost(order[0][0]) if self.policy == "srpt" else float("inf")
        take, taken = [], set()
        for item in order:
            if len(take) >= self.ppl:
                break
            if self._group(item[0]) == g and self._point_cost(item[0]) <= cap:
                take.append(item)
                taken.add(id(item))
        self._pending = [it for it in self._pending if id(it) not in taken]
        return take

    def _lane_loop(self, lane):
        ctx = self.lanes[lane]
        precision = int(getattr(ctx, "options", {}).get("precision", 0))   # the lane's current option
        while True:
            with self._cv:
                while not self._stop and not self._pending:
                    self._cv.wait(timeout=0.05)
                if self._stop and not self._pending:
                    return
                batch = self._take_batch()
                ids = np.array([self._resident[self._key(r)].ids[lane] for r, _ in batch], dtype=np.int32)
            req0 = batch[0][0]
            E = np.array([r.energies[i] for r, i in batch])
            try:
                if int(req0.precision) != precision:
                    ctx.update_options(precision=int(req0.precision))
                    precision = int(req0.precision)
                T, led, nc, st = ctx.transmissions(ids, E, req0.pairs, eta=req0.eta, ldos=req0.ldos,
                                                   dos_delta=req0.dos_delta, check=False)
                err = None
            except Exception as exc:                       # a call error fails the batch's points
                T, led, nc, st = None, None, None, None
                err = str(exc)
            with self._cv:
                for q, (r, i) in enumerate(batch):
                    if err is None:
                        r.T[i] = T[q]
                        r.ncyc[i] = nc[q]
                        r.status[i] = st[q]
                        if r.ldos:
                            if r.ledos is None:
                                r.ledos = np.zeros((r.energies.size, led.shape[1]))
                            r.ledos[i] = led[q, :r.ledos.shape[1]]
                    else:
                        r.status[i] = native.CUDA
                        r.error = err
                    r._left -= 1
                    if r._left == 0:
                        self._finish(r)
                self.points_done += len(batch)
                self.launches += 1
                self._cv.notify_all()

    def _finish(self, r):
        r.t_done = time.perf_counter()
        k = self._key(r)
        active = any(x is r for x in self._active)
        if k in self._resident and active:
            self._resident[k].users -= 1
            self._resident[k].last_use = r.t_done
        if active:
            self._active = [x for x in self._active if x is not r]
        self.completed.append(r)
        r._done.set()
