"""Schedule autotuner for transmission and DOS solves.

The engine's tile shapes are fixed by its register and shared-memory budget
(64 x 64 product tiles, 16-column inversion leaves); what changes the speed
for a given device shape is the schedule:

- the persistent engine (options.schedule = 1) with 2 resident CTAs per SM
  (one CTA's latency-bound inversion steps overlap the other's products) or
  1 (a CTA gets the whole L2 share and tensor pipe of an SM);
- lock step (options.schedule = 2; 2-contact transmission, n <= 32): every
  point through each batched block operation at once, one CTA per point.

`tune` times each candidate that the device shape admits on a sample of the
caller's own points, applies the fastest on top of the caller's other
options, and remembers it per device shape (optionally in a JSON file), so
later calls with the same shape skip the search.  Every candidate computes
the reference's operation sequence in complex FP64: the engine's CTA counts
give identical bits, lock step differs from them in the last bits
(summation order).
"""
from __future__ import annotations

import json
import os
import time
from typing import Dict, Optional, Sequence

import numpy as np

_CACHE: Dict[str, dict] = {}

# candidate schedules, in the order they are tried
ENGINE_2 = {"schedule": 1, "ctas_per_sm": 2}
ENGINE_1 = {"schedule": 1, "ctas_per_sm": 1}
LOCKSTEP = {"schedule": 2, "ctas_per_sm": 0}


def shape_key(dev, mode: str) -> str:
    """Devices with the same block structure share a schedule."""
    return "%s:nbl=%d:nmax=%d:ncont=%d:norb=%d" % (mode, dev.nbl, max(dev.pl_size + dev.lead_size), dev.ncont,
                                                    dev.norb)


def _name(c: dict) -> str:
    return "lockstep" if c["schedule"] == 2 else "engine_%d" % c["ctas_per_sm"]


def _time_call(fn, repeats: int) -> float:
    best = float("inf")
    for _ in range(repeats):
        t0 = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t0)
    return best


def tune(ctx, device_id: int, energies: Sequence[float], mode: str = "T", eta: float = 1e-4,
         candidates: Sequence[dict] = (ENGINE_2, ENGINE_1, LOCKSTEP), repeats: int = 1,
         cache_file: Optional[str] = None) -> dict:
    """Picks the schedule for this device shape by timing the candidates on
    `energies` (a sample: a few times the number of SMs is enough) and
    applies it to `ctx` on top of the options already set there.  mode "T"
    times the transmission solve, "DOS" the transmission + DOS solve; a
    candidate the shape or mode does not admit (lock step for DOS, for n >
    32, for contacts off blocks 1 and nbl) is skipped.  Returns the record
    {"schedule", "ctas_per_sm", "choice", "timings", "key"}."""
    from . import native
    dev = ctx.devices[device_id]
    key = shape_key(dev, mode)
    if cache_file and not _CACHE and os.path.exists(cache_file):
        with open(cache_file) as f:
            _CACHE.update(json.load(f))
    rec = _CACHE.get(key)
    base = {k: v for k, v in ctx.options.items() if k not in ("schedule", "ctas_per_sm")}
    if rec is None:
        E = np.ascontiguousarray(energies, dtype=np.float64)
        if mode == "DOS":
            call = lambda: ctx.transmission_dos(device_id, E, eta=eta, check=False)
        else:
            call = lambda: ctx.transmission(device_id, E, eta=eta, check=False)
        timings = {}
        try:
            for c in candidates:
                ctx.set_options(**base, **c)
                try:
                    call()                                # workspace growth and first-touch outside the timing
                except native.NegfError as e:
                    if e.code != native.BAD_ARG:
                        raise
                    continue                              # not admitted for this shape or mode
                timings[_name(c)] = (c, _time_call(call, repeats))
        finally:
            ctx.set_options(**base)
        best = min(timings, key=lambda k: timings[k][1])
        c = timings[best][0]
        rec = {"schedule": c["schedule"], "ctas_per_sm": c["ctas_per_sm"], "choice": best,
               "timings": {k: v[1] for k, v in timings.items()}, "key": key}
        _CACHE[key] = rec
        if cache_file:
            with open(cache_file, "w") as f:
                json.dump(_CACHE, f, indent=1)
    ctx.set_options(**base, schedule=int(rec["schedule"]), ctas_per_sm=int(rec["ctas_per_sm"]))
    return rec


def forget():
    _CACHE.clear()
