"""GPU parity of the row-wise Fftm (forward, inverse with scale) through the C ABI
against the FP64 oracle, the reference's golden vectors and the reference
library's own outputs.  Tolerance: relative L2 <= 2e-6 against FP64, and the
reference's own metric test::diff < -100 dB."""
import numpy as np
import pytest

from conftest import crandn
from openvsip_b200 import FcbError, Fftm, fft_fwd, fft_inv

pytestmark = pytest.mark.gpu
RTOL = 2e-6


def _torch():
    import torch
    return torch


@pytest.mark.parametrize("logn", range(0, 17))
def test_fftm_forward_inverse_vs_fp64(oracle, logn):
    n = 1 << logn
    rows = max(3, min(64, (1 << 20) // n))
    rng = np.random.default_rng(100 + logn)
    x = (rng.uniform(-1, 1, (rows, n)) + 1j * rng.uniform(-1, 1, (rows, n))).astype(np.complex64)
    fwd = Fftm(rows, n, fft_fwd, 1.0)
    inv = Fftm(rows, n, fft_inv, 1.0 / n)
    X = fwd(x)
    want = oracle.fft_rows(x, -1)
    assert oracle.rel_l2(X, want) <= RTOL, (n, oracle.rel_l2(X, want))
    y = inv(x)
    want_i = oracle.fft_rows(x, +1, 1.0 / n)
    assert oracle.rel_l2(y, want_i) <= RTOL, (n, oracle.rel_l2(y, want_i))
    # round trip (the reference's tests/fftm.cpp forward/inverse pairing)
    xr = inv(X)
    assert oracle.rel_l2(xr, x) <= RTOL


@pytest.mark.parametrize("k", range(1, 9))
def test_fftm_reference_golden_vectors(oracle, golden_fft_ext, k):
    x = golden_fft_ext[f"f{k}_in"].astype(np.complex64)[None, :]
    want = golden_fft_ext[f"f{k}_out"]
    scale = float(golden_fft_ext[f"f{k}_scale"])
    n = x.shape[1]  # f2 (768) and f4 (19) take the Bluestein path
    got = Fftm(1, n, fft_fwd, scale)(x)[0]
    assert oracle.error_db(want, got) < -100


@pytest.mark.parametrize("n", [64, 128, 256, 512])
def test_fftm_matches_reference_library(oracle, golden_ref, n):
    x = golden_ref[f"fftm_in_{n}"]
    f = Fftm(5, n, fft_fwd, 1.0)(x)
    i = Fftm(5, n, fft_inv, 1.0 / n)(x)
    assert oracle.error_db(golden_ref[f"fftm_fwd_{n}"], f) < -100
    assert oracle.error_db(golden_ref[f"fftm_inv_{n}"], i) < -100


def test_fftm_host_device_inplace_strided_fewer_rows(oracle):
    torch = _torch()
    n, rows = 4096, 40
    rng = np.random.default_rng(5)
    big = crandn(rng, (rows, n + 64))
    x = big[:, :n]  # row stride n + 64
    f = Fftm(rows + 8, n, fft_fwd, 2.0)  # planned for more rows than used
    host = f(x)
    want = 2.0 * oracle.fft_rows(x, -1)
    assert oracle.rel_l2(host, want) <= RTOL
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dev = f(dx)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dev.cpu().numpy(), host)  # same kernels -> bit-identical
    f.in_place(dx)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dx.cpu().numpy(), host)
    with pytest.raises(FcbError):
        f(crandn(rng, (rows + 9, n)))  # more rows than planned


@pytest.mark.parametrize("n", [1024, 16384, 65536])
def test_fftm_accuracy_vs_fp32_cpu_fft(oracle, n):
    # "no worse than 2x the FP32 CPU FFT": scipy's pocketfft complex64 stands in
    # for FFTW3's FP32 path, which is not installed.
    import scipy.fft
    rng = np.random.default_rng(n)
    x = crandn(rng, (16, n))
    ref = oracle.fft_rows(x, -1)
    cpu = scipy.fft.fft(x, axis=1)
    assert cpu.dtype == np.complex64
    gpu = Fftm(16, n, fft_fwd, 1.0)(x)
    assert oracle.rel_l2(gpu, ref) <= 2 * oracle.rel_l2(cpu, ref) + 1e-9


@pytest.mark.parametrize("threads", [-256, 512, 256])
def test_every_variant_at_16384(oracle, threads):
    # all kernel variants of 16384-sample rows, forward, inverse and fused
    # (-256: 256 threads x 64 samples, 3 stages; the others 32 samples, 4
    # stages; 256: a cluster of two CTAs)
    from openvsip_b200 import Fastconv, _lib
    lib = _lib.lib()
    n, rows = 16384, 24
    saved = [lib.fcb_tune_get(n, k) for k in range(3)]
    try:
        for k in range(3):
            _lib.check(lib.fcb_tune_set(n, k, threads))
        rng = np.random.default_rng(700 + threads)
        x = crandn(rng, (rows, n))
        rep = crandn(rng, (n,))
        f = Fftm(rows, n, fft_fwd, 1.0)
        assert f.info()["threads"] == abs(threads)
        assert oracle.rel_l2(f(x), oracle.fft_rows(x, -1)) <= RTOL
        assert oracle.rel_l2(Fftm(rows, n, fft_inv, 1.0 / n)(x), oracle.fft_rows(x, +1, 1.0 / n)) <= RTOL
        w = crandn(rng, (rows, n))
        assert oracle.rel_l2(Fastconv(rep, rows)(x), oracle.fastconv(x, rep)) <= RTOL
        assert oracle.rel_l2(Fastconv(w, rows)(x), oracle.fastconv(x, w)) <= RTOL
    finally:
        for k in range(3):
            _lib.check(lib.fcb_tune_set(n, k, saved[k]))
