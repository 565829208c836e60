"""negf_b200_decimation_noalloc, the decimation entry point that allocates no
device memory (its scratch is a fixed array compiled into the library), for
callers that cannot allocate: codes whose device memory belongs to another
allocator, and loops that cannot afford the device synchronisation of
cudaMalloc/cudaFree.  Its output must equal the work-buffer entry point's
(negf_b200_decimation_batched) on two calls in a row, the second one reusing
the scratch the first left behind.  This file is collected last."""
import numpy as np
import pytest

from libnegf_b200 import generators as G
from libnegf_b200 import native

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _problem(n, energies, seed):
    dev = G.transport_c0(nbl=3, n=n, seed=seed)
    Ao, Bo, Co = [], [], []
    for e in energies:
        Ec = e + 1e-6j
        Ao.append(Ec * np.eye(n) - dev.lead_h00[1])
        Bo.append(-dev.lead_h01[1])
        Co.append(-dev.lead_h01[1].conj().T)
    dev_t = lambda a: torch.from_numpy(np.ascontiguousarray(np.array(a).transpose(0, 2, 1))).cuda()
    return dev_t(Ao), dev_t(Bo), dev_t(Co)


def _run_batched(L, n, b, Ao, Bo, Co):
    Go = torch.empty_like(Ao)
    nc = torch.zeros(b, dtype=torch.int32, device="cuda")
    work = torch.empty(L.negf_b200_decimation_work_bytes(b, n), dtype=torch.uint8, device="cuda")
    rc = L.negf_b200_decimation_batched(b, n, Ao.data_ptr(), Bo.data_ptr(), Co.data_ptr(), Go.data_ptr(),
                                        nc.data_ptr(), 1e-9, 300, work.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    return Go.cpu().numpy(), nc.cpu().numpy()


def _run_noalloc(L, n, b, Ao, Bo, Co):
    Go = torch.full_like(Ao, float("nan"))
    nc = torch.zeros(b, dtype=torch.int32, device="cuda")
    rc = L.negf_b200_decimation_noalloc(b, n, Ao.data_ptr(), Bo.data_ptr(), Co.data_ptr(), Go.data_ptr(),
                                        nc.data_ptr(), 1e-9, 300, None)
    torch.cuda.synchronize()
    assert rc == 0
    return Go.cpu().numpy(), nc.cpu().numpy()


def test_noalloc_decimation_matches_batched_on_two_calls():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = native.load()
    cases = [(32, [-1.3, 0.2, 2.2], 4), (96, [0.7, -0.4], 9)]   # second call: other order and batch
    for n, Es, seed in cases:
        b = len(Es)
        Ao, Bo, Co = _problem(n, Es, seed)
        g_ref, nc_ref = _run_batched(L, n, b, Ao, Bo, Co)
        g, nc = _run_noalloc(L, n, b, Ao, Bo, Co)
        assert np.all(nc == nc_ref)
        scale = max(1.0, np.abs(g_ref).max())
        assert np.isfinite(g).all()
        assert np.abs(g - g_ref).max() <= 1e-9 * scale


def test_noalloc_calls_leave_free_device_memory_unchanged():
    """After a first call (which loads the module and resolves the array's
    address), further calls change the device's free memory by nothing: the
    scratch is the fixed array, not an allocation."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = native.load()
    n, Es = 64, [-1.1, 0.3, 1.7]
    b = len(Es)
    Ao, Bo, Co = _problem(n, Es, 5)
    Go = torch.empty_like(Ao)
    nc = torch.zeros(b, dtype=torch.int32, device="cuda")
    call = lambda: L.negf_b200_decimation_noalloc(b, n, Ao.data_ptr(), Bo.data_ptr(), Co.data_ptr(),
                                                  Go.data_ptr(), nc.data_ptr(), 1e-9, 300, None)
    assert call() == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        assert call() == 0
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_requests_beyond_the_fixed_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = native.load()
    n, b = 512, 64   # 64 * 15 * 512^2 * 16 bytes = 4 GiB > 64 MiB
    Ao = torch.zeros((1, n, n), dtype=torch.complex128, device="cuda")
    Go = torch.zeros_like(Ao)
    rc = L.negf_b200_decimation_noalloc(b, n, Ao.data_ptr(), Ao.data_ptr(), Ao.data_ptr(), Go.data_ptr(),
                                        None, 1e-9, 300, None)
    assert rc == native.ADMISSION
