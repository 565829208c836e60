"""The complex product on the integer tensor cores (negf_b200_zgemm_batched_i8:
int8 digit splitting, tcgen05 kind::i8, TMEM accumulators) against complex128
products: numpy's (BLAS zgemm) and the FP64 tensor-core product of this
library (negf_b200_zgemm_batched).

Bound per element: the splitting keeps every operand element to within
2^(e - 7 slices) of its value (e: the row's (A) or column's (B) power-of-two
scale) and drops the digit pairs of level min(slices + 1, 8) and below, each
at most slices 2^(-7 level) of the scale, so
|C - AB| <= 2K (2 2^(-7 slices) + 1.01 slices 2^(-7 levels)) 2^(eA_r + eB_c),
plus the FP64 rounding of the reference product."""

import ctypes

import numpy as np
import pytest

from libnegf_b200 import native

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _bound_factor(k, slices):
    levels = min(slices + 1, 8)
    return 2 * k * (2 * 2.0 ** (-7 * slices) + 1.01 * slices * 2.0 ** (-7 * levels))


def _rand(rng, shape, spread=False):
    z = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    if spread:   # rows and columns of very different size
        z = z * np.exp(rng.uniform(-8, 8, shape[:-1] + (1,))) * np.exp(rng.uniform(-4, 4, shape[:-2] + (1, shape[-1])))
    return z


def _dev(a):
    flat = np.ascontiguousarray(np.asarray(a, dtype=np.complex128).transpose(0, 2, 1))   # column-major per item
    return torch.from_numpy(flat).cuda()


def _host(t, rows, cols):
    return t.cpu().numpy().transpose(0, 2, 1).reshape(-1, rows, cols)


def _scale_exp(x, axis):
    mx = np.maximum(np.abs(x.real), np.abs(x.imag)).max(axis=axis)
    _, e = np.frexp(mx)
    return np.where(mx > 0, e, 0)


def run_i8(A, B, C0, alpha, beta, slices, status=False):
    L = native.load()
    b, m, k = A.shape
    n = B.shape[2]
    dA, dB, dC = _dev(A), _dev(B), _dev(C0)
    wb = L.negf_b200_zgemm_i8_work_bytes(b, m, n, k, slices)
    work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    st = torch.zeros(b, dtype=torch.int32, device="cuda")
    dp = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    al, be = np.array([alpha.real, alpha.imag]), np.array([beta.real, beta.imag])
    rc = L.negf_b200_zgemm_batched_i8(b, m, n, k, dp(al), dA.data_ptr(), 2 * m * k, dB.data_ptr(), 2 * k * n,
                                      dp(be), dC.data_ptr(), 2 * m * n, slices, work.data_ptr(), st.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    out = _host(dC, m, n)
    return (out, st.cpu().numpy()) if status else out


@pytest.mark.parametrize("b,m,n,k", [(1, 128, 64, 64), (1, 128, 128, 128), (3, 256, 256, 256), (2, 512, 512, 512),
                                     (2, 100, 70, 90), (3, 17, 33, 65), (1, 64, 192, 1024), (2, 1, 1, 1)])
@pytest.mark.parametrize("slices", [7])
def test_i8_product_against_complex128(b, m, n, k, slices):
    rng = np.random.default_rng(m * 7 + n * 3 + k + b)
    A, B, C0 = _rand(rng, (b, m, k)), _rand(rng, (b, k, n)), _rand(rng, (b, m, n))
    alpha, beta = 0.7 - 0.3j, 0.25 + 0.5j
    got = run_i8(A, B, C0, alpha, beta, slices)
    ref = alpha * (A @ B) + beta * C0
    for i in range(b):
        sc = np.ldexp(1.0, _scale_exp(A[i], 1)[:, None] + _scale_exp(B[i], 0)[None, :])
        bound = abs(alpha) * _bound_factor(k, slices) * sc + 1e-14 * np.abs(ref[i]).max()
        assert np.all(np.abs(got[i] - ref[i]) <= bound)
        # typical accuracy: like an FP64 product
        rel = np.abs(got[i] - ref[i]).max() / np.abs(ref[i]).max()
        assert rel < 2e-14, rel


@pytest.mark.parametrize("slices", [4, 5, 6, 7, 8])
def test_i8_error_falls_by_2_to_the_7_per_slice(slices):
    rng = np.random.default_rng(slices)
    A, B = _rand(rng, (1, 256, 256)), _rand(rng, (1, 256, 256))
    got = run_i8(A, B, np.zeros((1, 256, 256)), 1.0 + 0j, 0j, slices)
    ref = A @ B
    sc = np.ldexp(1.0, _scale_exp(A[0], 1)[:, None] + _scale_exp(B[0], 0)[None, :])
    err = np.abs(got[0] - ref[0])
    assert np.all(err <= _bound_factor(256, slices) * sc + 1e-14 * np.abs(ref).max())
    if slices <= 6:   # above FP64 rounding: the splitting error is what is seen
        assert (err / sc).max() > 2.0 ** (-7 * slices - 8)


def test_i8_rows_and_columns_of_different_scale():
    """Each row of A and column of B has its own exponent: elements 1e-7 and
    1e+7 apart keep their relative accuracy per row / column scale."""
    rng = np.random.default_rng(5)
    A, B = _rand(rng, (2, 256, 256), spread=True), _rand(rng, (2, 256, 256), spread=True)
    got = run_i8(A, B, np.zeros((2, 256, 256)), 1.0 + 0j, 0j, 7)
    ref = A @ B
    for i in range(2):
        sc = np.ldexp(1.0, _scale_exp(A[i], 1)[:, None] + _scale_exp(B[i], 0)[None, :])
        assert np.all(np.abs(got[i] - ref[i]) <= _bound_factor(256, 7) * sc + 1e-14 * np.abs(ref[i]))


def test_i8_matches_fp64_tensor_product():
    rng = np.random.default_rng(11)
    b, n = 4, 256
    A, B = _rand(rng, (b, n, n)), _rand(rng, (b, n, n))
    got = run_i8(A, B, np.zeros((b, n, n)), 1.0 + 0j, 0j, 7)
    L = native.load()
    dA, dB, dC = _dev(A), _dev(B), _dev(np.zeros((b, n, n)))
    dp = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    rc = L.negf_b200_zgemm_batched(b, n, n, n, dp(np.array([1.0, 0.0])), dA.data_ptr(), 2 * n * n, dB.data_ptr(),
                                   2 * n * n, dp(np.array([0.0, 0.0])), dC.data_ptr(), 2 * n * n, 0, None)
    torch.cuda.synchronize()
    assert rc == 0
    f64 = _host(dC, n, n)
    ref = A @ B
    e_i8 = np.abs(got - ref).max() / np.abs(ref).max()
    e_64 = np.abs(f64 - ref).max() / np.abs(ref).max()
    assert e_i8 < 20 * max(e_64, 1e-16), (e_i8, e_64)


def test_i8_in_place_and_nonfinite():
    rng = np.random.default_rng(3)
    A, B = _rand(rng, (2, 128, 128)), _rand(rng, (2, 128, 128))
    A[1, 5, 7] = np.nan
    C0 = _rand(rng, (2, 128, 128))
    got, st = run_i8(A, B, C0, -1.0 + 0j, 1.0 + 0j, 7, status=True)   # C = C0 - A B
    ref = C0[0] - A[0] @ B[0]
    assert np.abs(got[0] - ref).max() <= 1e-12 * np.abs(ref).max()
    assert st[0] == native.OK and st[1] == native.NONFINITE
    assert np.isnan(got[1]).all()
