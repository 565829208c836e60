"""Launch-shape autotuner for the persistent engine.

The engine's tile shapes are fixed by its register and shared-memory budget
(64 x 64 product tiles, 16-column inversion leaves); what changes the speed
for a given device is the launch schedule: resident CTAs per SM (2 overlaps
one CTA's latency-bound inversion steps with the other's products; 1 gives a
CTA the whole L2 share and tensor pipe of an SM) and how many points one
launch takes.  `tune` times each candidate on a sample of the caller's own
points, applies the fastest, and remembers it per device shape (optionally
in a JSON file), so later calls with the same shape skip the search.
"""
from __future__ import annotations

import json
import os
import time
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

_CACHE: Dict[str, dict] = {}


def shape_key(dev, mode: str) -> str:
    """Devices with the same block structure share a schedule."""
    return "%s:nbl=%d:nmax=%d:ncont=%d:norb=%d" % (mode, dev.nbl, max(dev.pl_size + dev.lead_size), dev.ncont,
                                                    dev.norb)


def _time_call(fn, repeats: int) -> float:
    best = float("inf")
    for _ in range(repeats):
        t0 = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t0)
    return best


def tune(ctx, device_id: int, energies: Sequence[float], mode: str = "T", eta: float = 1e-4,
         candidates: Sequence[int] = (2, 1), repeats: int = 1, cache_file: Optional[str] = None) -> dict:
    """Picks ctas_per_sm for this device shape by timing the candidates on
    `energies` (a sample: a few times the number of SMs is enough) and
    applies it to `ctx`.  mode "T" times the transmission solve, "DOS" the
    transmission + DOS solve.  Returns the record {"ctas_per_sm", "timings",
    "key"}."""
    dev = ctx.devices[device_id]
    key = shape_key(dev, mode)
    if cache_file and not _CACHE and os.path.exists(cache_file):
        with open(cache_file) as f:
            _CACHE.update(json.load(f))
    rec = _CACHE.get(key)
    if rec is None:
        E = np.ascontiguousarray(energies, dtype=np.float64)
        if mode == "DOS":
            call = lambda: ctx.transmission_dos(device_id, E, eta=eta, check=False)
        else:
            call = lambda: ctx.transmission(device_id, E, eta=eta, check=False)
        timings = {}
        for c in candidates:
            ctx.set_options(ctas_per_sm=int(c))
            call()                                    # workspace growth and first-touch outside the timing
            timings[int(c)] = _time_call(call, repeats)
        best = min(timings, key=timings.get)
        rec = {"ctas_per_sm": best, "timings": {str(k): v for k, v in timings.items()}, "key": key}
        _CACHE[key] = rec
        if cache_file:
            with open(cache_file, "w") as f:
                json.dump(_CACHE, f, indent=1)
    ctx.set_options(ctas_per_sm=int(rec["ctas_per_sm"]))
    return rec


def forget():
    _CACHE.clear()
