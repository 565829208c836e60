"""Multi-rank path on CPU: two gloo ranks shard a point list round robin,
solve their share, and the sum reduction of the scattered rows rebuilds the
single-rank result; the timing reduction takes the slowest rank.  The
per-point "solve" here is a host function: the sharding and the collectives
are what is under test (the GPU solve itself has its own parity tests)."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_solve(E):
    return np.stack([np.cos(3 * E) ** 2, np.sin(E) ** 2], axis=1)   # npts x npairs


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from libnegf_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        E = np.linspace(-2, 2, 37)
        idx = shard.shard_points(E.size, rank, world)
        rows = _fake_solve(E[idx])
        full = shard.reduce_rows(shard.scatter_rows(rows, idx, E.size), dist)
        # complex rows (density / Gn blocks) keep their imaginary part
        crow = rows[:, :1] * np.exp(1j * E[idx])[:, None]
        cfull = shard.reduce_rows(shard.scatter_rows(crow, idx, E.size), dist)
        t = shard.max_over_ranks(1.0 + rank, dist)
        out[rank] = (full, t, idx.tolist(), cfull)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_rebuild_the_single_rank_result():
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    E = np.linspace(-2, 2, 37)
    ref = _fake_solve(E)
    cref = ref[:, :1] * np.exp(1j * E)[:, None]
    for r in range(world):
        full, t, idx, cfull = out[r]
        assert np.array_equal(full, ref)
        assert cfull.dtype == np.complex128 and np.array_equal(cfull, cref)
        assert t == float(world)               # the slowest rank's time
    assert sorted(out[0][2] + out[1][2]) == list(range(E.size))


def test_shard_points_single_rank_and_bad_args():
    from libnegf_b200 import shard
    assert shard.shard_points(5).tolist() == [0, 1, 2, 3, 4]
    assert shard.shard_points(7, 2, 3).tolist() == [2, 5]
    with pytest.raises(ValueError):
        shard.shard_points(4, 3, 3)
