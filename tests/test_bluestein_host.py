"""CPU check of the Bluestein decomposition that the GPU plans for
non-power-of-two rows use, restated in FP64 numpy step by step as the device
code runs it (chirp, zero-padded pre-multiply, circular convolution of the
work rows through a power-of-two FFT with the replica FFT(b) and the 1/M of the
fused pass, post-multiply; the fast convolution with the chirps cancelled
between its two passes).  It pins the signs, the filter layout and the work
length M = next power of two >= 2N - 1 against numpy's FFT."""
import numpy as np
import pytest


def _work_len(n):
    m = 1
    while m < 2 * n - 1:
        m <<= 1
    return m


def _chirp(n, sign):
    k = np.arange(n, dtype=np.int64)
    return np.exp(1j * np.pi * sign * ((k * k) % (2 * n)) / n)


def _filter(n, m, sign):
    c = np.conj(_chirp(n, sign))
    b = np.zeros(m, dtype=np.complex128)
    b[:n] = c
    b[m - n + 1:] = c[1:][::-1]
    return b


def _fused(a, spec):
    """The fused pass: IFFT_M(FFT_M(a) * spec / M) * M / M (replica table holds spec / M)."""
    m = a.shape[-1]
    return np.fft.ifft(np.fft.fft(a, axis=-1) * (spec / m), axis=-1) * m


def _bluestein_rows(x, sign, scale=1.0):
    rows, n = x.shape
    m = _work_len(n)
    c = _chirp(n, sign)
    spec = np.fft.fft(_filter(n, m, sign))
    a = np.zeros((rows, m), dtype=np.complex128)
    a[:, :n] = x * c
    y = _fused(a, spec)
    return scale * c * y[:, :n]


@pytest.mark.parametrize("n", [3, 5, 6, 18, 19, 68, 252, 768, 1000, 4095])
@pytest.mark.parametrize("sign", [-1, +1])
def test_bluestein_rows_match_fft(n, sign):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((3, n)) + 1j * rng.standard_normal((3, n))
    got = _bluestein_rows(x, sign)
    want = np.fft.fft(x, axis=1) if sign < 0 else np.fft.ifft(x, axis=1) * n
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-12


@pytest.mark.parametrize("n", [5, 68, 768, 1000])
def test_bluestein_fastconv_chirps_cancel(n):
    rng = np.random.default_rng(7 * n)
    x = rng.standard_normal((4, n)) + 1j * rng.standard_normal((4, n))
    r = rng.standard_normal((4, n)) + 1j * rng.standard_normal((4, n))
    m = _work_len(n)
    cf, ci = _chirp(n, -1), _chirp(n, +1)
    assert np.allclose(cf * ci, 1.0)
    sf, si = np.fft.fft(_filter(n, m, -1)), np.fft.fft(_filter(n, m, +1))
    a = np.zeros((4, m), dtype=np.complex128)
    a[:, :n] = x * cf
    y = _fused(a, sf)
    y[:, :n] *= r / n  # replica spectrum / n; the chirps cancel
    y[:, n:] = 0
    out = ci * _fused(y, si)[:, :n]
    want = np.fft.ifft(np.fft.fft(x, axis=1) * r, axis=1)
    assert np.linalg.norm(out - want) / np.linalg.norm(want) < 1e-12


def test_work_lengths_stay_within_the_fused_kernel():
    assert _work_len(3) == 8 and _work_len(768) == 2048 and _work_len(19) == 64
    assert _work_len(32767) == 65536 and _work_len(32768) == 65536
