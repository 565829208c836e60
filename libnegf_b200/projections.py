"""Projection index sets of the transmission and LDOS outputs.

libNEGF keeps two projections on its `Tnegf` object:

- `tun_proj`: orbital indices (1-based, global) over which the
  transmission trace runs; `get_tun_mask` (src/iterative_cpu.F90:586-618)
  turns them into a mask of the contact block's diagonal.  No indices = the
  whole trace.
- `dos_proj`: a list of orbital index sets (1-based); the LDOS of set k is
  the sum of -Im Gr_ii / pi over its indices (src/iterative.F90:1931-1945).

These helpers give the flat arrays the C-ABI takes.
"""
from __future__ import annotations

import numpy as np


def tun_mask(norb, tun_proj):
    """One byte per orbital (1 = inside the trace), or None for no projection."""
    if tun_proj is None:
        return None
    idx = np.asarray(tun_proj, dtype=np.int64).ravel()
    mask = np.zeros(norb, dtype=np.uint8)
    ok = (idx >= 1) & (idx <= norb)
    mask[idx[ok] - 1] = 1
    return mask


def tun_indices(tun_proj):
    """tun_proj as a contiguous int32 array of 1-based indices."""
    return np.ascontiguousarray(np.asarray(tun_proj, dtype=np.int32).ravel())


def dos_sets(dos_proj):
    """CSR form (ptr, idx) of a list of 1-based index sets: set k is
    idx[ptr[k]:ptr[k+1]], in the given order (repeated indices count again,
    as in the reference's accumulation loop)."""
    sets = [np.asarray(s, dtype=np.int32).ravel() for s in dos_proj]
    ptr = np.zeros(len(sets) + 1, dtype=np.int32)
    for k, s in enumerate(sets):
        ptr[k + 1] = ptr[k] + s.size
    idx = np.concatenate(sets).astype(np.int32) if sets and ptr[-1] > 0 else np.zeros(1, dtype=np.int32)
    return np.ascontiguousarray(ptr), np.ascontiguousarray(idx)
