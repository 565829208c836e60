"""Point sharding across ranks (one process per GPU).

(E, k) points are independent for T, DOS and the elastic-dephasing SCBA, so
ranks split the point list with no data-path collective and combine only the
per-point outputs at the end, as libNEGF does over MPI: energy points dealt
round robin (tunneling_int_def, src/integrations.F90:1649-1654), rows of the
result matrices owned by other ranks left at zero, then a sum reduction
(mpifx_reduceip, src/integrations.F90:1940-1941).  The process group is
torch.distributed's (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def shard_points(npts: int, rank: int = 0, world: int = 1) -> np.ndarray:
    """0-based indices of the points rank `rank` solves (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank %d of %d" % (rank, world))
    return np.arange(rank, npts, world, dtype=np.int64)


def scatter_rows(local_rows: np.ndarray, idx: np.ndarray, npts: int) -> np.ndarray:
    """Full-size matrix holding this rank's rows at their grid positions and
    zeros elsewhere (the layout the sum reduction expects)."""
    local_rows = np.asarray(local_rows)
    full = np.zeros((npts,) + local_rows.shape[1:], dtype=local_rows.dtype)
    full[idx] = local_rows
    return full


def reduce_rows(full: np.ndarray, dist=None) -> np.ndarray:
    """Sum of every rank's scatter_rows() matrix (all ranks get the result).
    Complex rows (density or Gn blocks) keep their imaginary part: they are
    reduced as their float64 (re, im) pairs and viewed back."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return full
    import torch
    full = np.asarray(full)
    cplx = np.iscomplexobj(full)
    flat = (np.ascontiguousarray(full, dtype=np.complex128).view(np.float64) if cplx
            else np.ascontiguousarray(full, dtype=np.float64))
    t = torch.from_numpy(flat.copy())
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    out = t.cpu().numpy()
    return out.view(np.complex128) if cplx else out


def max_over_ranks(value: float, dist=None) -> float:
    """The largest `value` over ranks (a multi-GPU time is the slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
