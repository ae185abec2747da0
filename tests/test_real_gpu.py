"""GPU parity of the real-input Fftm (real -> complex forward, complex -> real
inverse; fftm_backend<float, complex<float>, A, fft_fwd> and
fftm_backend<complex<float>, float, A, fft_inv>) and of the column-axis Fftm,
against FP64 numpy: relative L2 <= 2e-6.  Sizes include the reference's own
real test lengths (tests/fftm.cpp test_real: 16, 128, 242 along columns),
odd lengths, unaligned row strides and host / device data."""
import numpy as np
import pytest

from conftest import crandn
from openvsip_b200 import FcbError, Fftm, FftmReal, col, fft_fwd, fft_inv, row

pytestmark = pytest.mark.gpu
RTOL = 2e-6


def _rel(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


SIZES = [2, 4, 16, 128, 242, 1000, 1024, 4096, 16384, 65536, 131072, 3, 125, 1001, 32767]


@pytest.mark.parametrize("n", SIZES)
def test_r2c_c2r_rows_vs_fp64(n):
    rows = max(2, min(32, (1 << 20) // n))
    rng = np.random.default_rng(500 + n)
    x = rng.standard_normal((rows, n)).astype(np.float32)
    X = FftmReal(rows, n, fft_fwd, 1.0)(x)
    assert X.shape == (rows, n // 2 + 1) and X.dtype == np.complex64
    want = np.fft.rfft(x.astype(np.float64), axis=1)
    assert _rel(X, want) <= RTOL, (n, _rel(X, want))
    # inverse of an arbitrary half spectrum (bins 0 and n/2 taken as real, like FFTW's c2r)
    H = crandn(rng, (rows, n // 2 + 1))
    y = FftmReal(rows, n, fft_inv, 1.0 / n)(H)
    assert y.shape == (rows, n) and y.dtype == np.float32
    Hr = H.astype(np.complex128)
    Hr[:, 0] = Hr[:, 0].real
    if n % 2 == 0:
        Hr[:, -1] = Hr[:, -1].real
    want_y = np.fft.irfft(Hr, n, axis=1)
    assert _rel(y, want_y) <= RTOL, (n, _rel(y, want_y))
    # round trip
    xr = FftmReal(rows, n, fft_inv, 1.0 / n)(X)
    assert _rel(xr, x) <= RTOL


@pytest.mark.parametrize("n", [16, 128, 242])
def test_reference_real_test_shapes_along_columns(n):
    # tests/fftm.cpp test_real: Fftm<T, complex<T>, col, fft_fwd>(Domain<2>(N, 5)) and back with 1/N
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, 5)).astype(np.float32)
    f = FftmReal(n, 5, fft_fwd, 1.0, axis=col)
    i = FftmReal(n, 5, fft_inv, 1.0 / n, axis=col)
    X = f(x)
    assert X.shape == (n // 2 + 1, 5)
    assert _rel(X, np.fft.rfft(x.astype(np.float64), axis=0)) <= RTOL
    assert _rel(i(X), x) <= RTOL


def test_real_unaligned_strides_host_and_device():
    import torch
    n, rows = 1000, 37
    rng = np.random.default_rng(3)
    big = rng.standard_normal((rows, n + 3)).astype(np.float32)
    x = big[:, 1:n + 1]  # odd row stride and a 4-byte offset: not 8-byte aligned
    f = FftmReal(rows, n, fft_fwd, 2.0)
    host = f(x)
    assert _rel(host, 2.0 * np.fft.rfft(x.astype(np.float64), axis=1)) <= RTOL
    dbig = torch.from_numpy(big).cuda()
    dev = f(dbig[:, 1:n + 1])
    torch.cuda.synchronize()
    np.testing.assert_allclose(dev.cpu().numpy(), host, rtol=0, atol=1e-3)
    # inverse into an unaligned real output
    H = crandn(rng, (rows, n // 2 + 1))
    out = np.zeros((rows, n + 3), dtype=np.float32)
    FftmReal(rows, n, fft_inv, 1.0)(H, out[:, 1:n + 1])
    Hr = H.astype(np.complex128)
    Hr[:, 0] = Hr[:, 0].real
    Hr[:, -1] = Hr[:, -1].real
    assert _rel(out[:, 1:n + 1], np.fft.irfft(Hr, n, axis=1) * n) <= RTOL
    assert not out[:, 0].any() and not out[:, -2:].any()  # nothing written outside the view


def test_real_rejects_bad_calls():
    with pytest.raises(FcbError):
        FftmReal(4, 65537 * 2 + 1, fft_fwd)  # odd beyond 32767
    f = FftmReal(4, 64, fft_fwd)
    with pytest.raises(TypeError):
        f(np.zeros((4, 64), dtype=np.complex64))  # r2c takes real input


@pytest.mark.parametrize("n,m", [(256, 7), (68, 5), (18, 3), (4096, 33)])
def test_fftm_along_columns(oracle, n, m):
    import torch
    # tests/fftm.cpp test_by_ref_y / test_by_val_y: Fftm<C, C, col, D>(Domain<2>(N, M))
    rng = np.random.default_rng(n + m)
    x = crandn(rng, (n, m))
    f = Fftm(n, m, fft_fwd, 1.0, axis=col)
    i = Fftm(n, m, fft_inv, 1.0 / n, axis=col)
    X = f(x)
    assert oracle.rel_l2(X, np.fft.fft(x.astype(np.complex128), axis=0)) <= RTOL
    assert oracle.rel_l2(i(X), x) <= RTOL
    dx = torch.from_numpy(x).cuda()
    dX = f(dx)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dX.cpu().numpy(), X)
    f.in_place(dx)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dx.cpu().numpy(), X)
    assert Fftm(n, m, fft_fwd, 1.0, axis=row)(x).shape == (n, m)
