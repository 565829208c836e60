"""Launch schedule: the autotuner's choice never changes results, and a
device-buffer solve captured into a CUDA graph replays to the same outputs."""
import ctypes

import numpy as np
import pytest

from libnegf_b200 import generators as G


@pytest.mark.gpu
def test_autotune_picks_a_schedule_without_changing_results(gpu_ctx, tmp_path):
    """The tuner times the engine at 2 and 1 CTAs per SM and lock step where
    the shape admits it, applies the fastest on top of the caller's options,
    and reads its choice back from the file.  The engine's CTA counts give
    identical bits; every schedule is at strict parity with the oracle."""
    from conftest import assert_T_strict, oracle_spread, xp_reference
    from libnegf_b200 import autotune
    from oracle import oracle as O
    dev = G.transport_c0(nbl=6, n=16, seed=2)
    E = np.linspace(-2, 2, 300)
    did = gpu_ctx.upload(dev)
    try:
        got = {}
        for name, c in (("engine_2", autotune.ENGINE_2), ("engine_1", autotune.ENGINE_1),
                        ("lockstep", autotune.LOCKSTEP)):
            gpu_ctx.set_options(sgf_tol=1e-10, **c)
            got[name] = gpu_ctx.transmission(did, E, eta=1e-4)
        assert np.array_equal(got["engine_1"][0], got["engine_2"][0])
        ref, spread = oracle_spread(lambda d: dict(zip(("T", "ncyc"), O.transmission(d, E, eta=1e-4,
                                                                                         sgf_tol=1e-10)[:2])),
                                    dev, nsamp=2)
        x = xp_reference(dev, E, 1e-4, sgf_tol=1e-10)
        for name, (T, nc, st) in got.items():
            assert np.array_equal(nc, ref["ncyc"]), name
            assert_T_strict(T, ref["T"], x, spread=spread["T"], what=name)
        gpu_ctx.set_options(sgf_tol=1e-10)
        autotune.forget()
        rec = autotune.tune(gpu_ctx, did, E[:200], mode="T", cache_file=str(tmp_path / "sched.json"))
        assert set(rec["timings"]) == {"engine_2", "engine_1", "lockstep"}
        assert gpu_ctx.options["sgf_tol"] == 1e-10                 # the caller's options stay
        assert np.array_equal(gpu_ctx.transmission(did, E, eta=1e-4)[0], got[rec["choice"]][0])
        autotune.forget()
        rec2 = autotune.tune(gpu_ctx, did, E[:200], mode="T", cache_file=str(tmp_path / "sched.json"))
        assert rec2 == rec                                   # read back from the file
        # the DOS solve has no lock step: only the engine's candidates
        autotune.forget()
        rec3 = autotune.tune(gpu_ctx, did, E[:200], mode="DOS")
        assert set(rec3["timings"]) == {"engine_2", "engine_1"} and rec3["schedule"] == 1
    finally:
        autotune.forget()
        gpu_ctx.set_options()
        gpu_ctx.release(did)


@pytest.mark.gpu
def test_device_solve_replays_from_a_cuda_graph(gpu_ctx):
    torch = pytest.importorskip("torch")
    from libnegf_b200 import native
    dev = G.transport_c0(nbl=5, n=8, seed=1)
    E = np.linspace(-2.5, 2.5, 64)
    did = gpu_ctx.upload(dev)
    L = native.load()
    try:
        n = E.size
        d_ids = torch.full((n,), did, dtype=torch.int32, device="cuda")
        d_E = torch.from_numpy(E).cuda()
        d_T = torch.zeros(n, dtype=torch.float64, device="cuda")
        d_dos = torch.zeros((n, dev.norb), dtype=torch.float64, device="cuda")
        d_nc = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_st = torch.zeros(n, dtype=torch.int32, device="cuda")
        s = torch.cuda.Stream()

        def call():
            return L.negf_b200_transmission_dos_dev(gpu_ctx.handle, n, d_ids.data_ptr(), d_E.data_ptr(), 1e-4, 1e-4,
                                                    1, 2, d_T.data_ptr(), d_dos.data_ptr(), dev.norb,
                                                    d_nc.data_ptr(), d_st.data_ptr(), ctypes.c_void_p(s.cuda_stream))
        with torch.cuda.stream(s):
            assert call() == 0                               # eager (sizes the workspace)
        torch.cuda.synchronize()
        T_eager, dos_eager = d_T.cpu().numpy().copy(), d_dos.cpu().numpy().copy()
        d_T.zero_(); d_dos.zero_()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            rc = call()
        assert rc == 0
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(d_T.cpu().numpy(), T_eager)
        assert np.array_equal(d_dos.cpu().numpy(), dos_eager)
        d_E.copy_(torch.from_numpy(E[::-1].copy()))           # new inputs, same graph
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(d_T.cpu().numpy(), T_eager[::-1])
        del g
    finally:
        gpu_ctx.release(did)


@pytest.mark.gpu
def test_large_host_read_back_matches_the_device_call(gpu_ctx):
    """A DOS result of 1 MiB or more reaches the caller's (pageable) array
    through the context's pinned staging buffer: bit for bit what the
    device-buffer call leaves on the device, on a first call (the buffer is
    allocated) and a second one into an array that already holds data."""
    torch = pytest.importorskip("torch")
    from libnegf_b200 import native
    dev = G.transport_c0(nbl=4, n=128, seed=3)
    E = np.linspace(-2.0, 2.0, 300)                   # 300 x 512 doubles = 1.2 MB of DOS
    did = gpu_ctx.upload(dev)
    L = native.load()
    try:
        n = E.size
        assert n * dev.norb * 8 >= 1 << 20
        gpu_ctx.set_options(schedule=1)
        d_ids = torch.full((n,), did, dtype=torch.int32, device="cuda")
        d_E = torch.from_numpy(E).cuda()
        d_T = torch.zeros(n, dtype=torch.float64, device="cuda")
        d_dos = torch.zeros((n, dev.norb), dtype=torch.float64, device="cuda")
        d_nc = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_st = torch.zeros(n, dtype=torch.int32, device="cuda")
        s = torch.cuda.Stream()
        rc = L.negf_b200_transmission_dos_dev(gpu_ctx.handle, n, d_ids.data_ptr(), d_E.data_ptr(), 1e-4, 1e-4, 1, 2,
                                              d_T.data_ptr(), d_dos.data_ptr(), dev.norb, d_nc.data_ptr(),
                                              d_st.data_ptr(), ctypes.c_void_p(s.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        T_dev, dos_dev = d_T.cpu().numpy(), d_dos.cpu().numpy()
        T1, dos1, nc1, st1 = gpu_ctx.transmission_dos(did, E, eta=1e-4, dos_delta=1e-4)
        assert np.array_equal(T1, T_dev) and np.array_equal(dos1, dos_dev)
        assert np.array_equal(nc1, d_nc.cpu().numpy()) and not st1.any()
        T2, dos2, _, _ = gpu_ctx.transmission_dos(did, E[::-1].copy(), eta=1e-4, dos_delta=1e-4)
        assert np.array_equal(T2, T_dev[::-1]) and np.array_equal(dos2, dos_dev[::-1])
    finally:
        gpu_ctx.set_options()
        gpu_ctx.release(did)
