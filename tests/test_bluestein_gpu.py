"""GPU parity of non-power-of-two rows (Bluestein through power-of-two work
rows) for Fftm and the fast convolution, against the FP64 oracle: relative L2
<= 2e-6, and no worse than twice the FP32 CPU FFT (pocketfft complex64) at the
same lengths.  The sizes include the reference's own test lengths
(tests/fftm.cpp: 18, 68, 252; tests/fft_ext/data: 19, 768)."""
import numpy as np
import pytest

from conftest import crandn
from openvsip_b200 import Fastconv, Fftm, fft_fwd, fft_inv, replica_spectrum

pytestmark = pytest.mark.gpu
RTOL = 2e-6
SIZES = [3, 5, 6, 18, 19, 68, 100, 252, 768, 1000, 3000, 4095, 12345, 24000, 32767]


@pytest.mark.parametrize("n", SIZES)
def test_fftm_non_pow2_vs_fp64(oracle, n):
    rows = max(2, min(40, (1 << 19) // n))
    rng = np.random.default_rng(300 + n)
    x = crandn(rng, (rows, n))
    X = Fftm(rows, n, fft_fwd, 1.0)(x)
    want = oracle.fft_rows(x, -1)
    assert oracle.rel_l2(X, want) <= RTOL, (n, oracle.rel_l2(X, want))
    y = Fftm(rows, n, fft_inv, 1.0 / n)(x)
    want_i = oracle.fft_rows(x, +1, 1.0 / n)
    assert oracle.rel_l2(y, want_i) <= RTOL, (n, oracle.rel_l2(y, want_i))
    xr = Fftm(rows, n, fft_inv, 1.0 / n)(X)
    assert oracle.rel_l2(xr, x) <= RTOL


@pytest.mark.parametrize("n", [18, 768, 1000, 12345])
def test_fftm_non_pow2_accuracy_vs_fp32_cpu_fft(oracle, n):
    import scipy.fft
    rng = np.random.default_rng(n)
    x = crandn(rng, (16, n))
    ref = oracle.fft_rows(x, -1)
    cpu = scipy.fft.fft(x, axis=1)
    assert cpu.dtype == np.complex64
    gpu = Fftm(16, n, fft_fwd, 1.0)(x)
    assert oracle.rel_l2(gpu, ref) <= 2 * oracle.rel_l2(cpu, ref) + 1e-9, (oracle.rel_l2(gpu, ref),
                                                                          oracle.rel_l2(cpu, ref))


def test_fftm_non_pow2_device_inplace_strided_and_chunks(oracle):
    import torch
    n, rows = 768, 50000  # 50000 rows x 2048-sample work rows: two work-buffer chunks
    rng = np.random.default_rng(9)
    big = crandn(rng, (rows, n + 8))
    x = big[:, :n]
    f = Fftm(rows, n, fft_fwd, 0.5)
    host = f(x)
    want = 0.5 * oracle.fft_rows(x[:4000], -1)
    assert oracle.rel_l2(host[:4000], want) <= RTOL
    assert oracle.rel_l2(host[-3000:], 0.5 * oracle.fft_rows(x[-3000:], -1)) <= RTOL
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dev = f(dx)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dev.cpu().numpy(), host)
    f.in_place(dx)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dx.cpu().numpy(), host)


@pytest.mark.parametrize("n", [5, 68, 768, 1000, 4095, 24000])
def test_fastconv_non_pow2_vs_fp64(oracle, n):
    rows = max(2, min(32, (1 << 19) // n))
    rng = np.random.default_rng(400 + n)
    x = crandn(rng, (rows, n))
    rep = crandn(rng, (n,))
    y = Fastconv(rep, rows)(x)
    assert oracle.rel_l2(y, oracle.fastconv(x, rep)) <= RTOL
    w = crandn(rng, (rows, n))  # matrix of coefficients
    yw = Fastconv(w, rows)(x)
    assert oracle.rel_l2(yw, oracle.fastconv(x, w)) <= RTOL


@pytest.mark.parametrize("n", [19, 768, 3000])
def test_fastconv_non_pow2_time_domain_replica(oracle, n):
    import torch
    chirp = oracle.lfm_chirp(n, 20.0, n).astype(np.complex64)
    want_spec = np.conj(np.fft.fft(chirp.astype(np.complex128)))
    spec = replica_spectrum(torch.from_numpy(chirp).cuda(), matched=True).cpu().numpy()
    assert oracle.rel_l2(spec, want_spec) <= 1e-7  # FP64 DFT, rounded once
    rng = np.random.default_rng(n)
    x = crandn(rng, (8, n))
    y = Fastconv(chirp, 8, kind="matched")(x)
    assert oracle.rel_l2(y, oracle.fastconv(x, want_spec.astype(np.complex64))) <= RTOL
