"""GPU parity of the fused fast convolution (forward Fftm -> vmmul<0> by the
replica spectrum -> inverse Fftm * 1/N) through the C ABI against the FP64
oracle and the reference library's own outputs.  Tolerance: relative L2 <=
2e-6 against FP64 (and test::diff < -100 dB where the reference tests use it)."""
import numpy as np
import pytest

from conftest import crandn
from openvsip_b200 import Fastconv, Fftm, fft_fwd, fft_inv, replica_spectrum, synth, vmmul

pytestmark = pytest.mark.gpu
RTOL = 2e-6


def _torch():
    import torch
    return torch


@pytest.mark.parametrize("logn", range(0, 17))
def test_fastconv_vs_fp64(oracle, logn):
    n = 1 << logn
    rows = max(3, min(64, (1 << 21) // n))
    rng = np.random.default_rng(200 + logn)
    x = crandn(rng, (rows, n))
    rep = crandn(rng, (n,))
    y = Fastconv(rep, rows)(x)
    want = oracle.fastconv(x, rep)
    assert oracle.rel_l2(y, want) <= RTOL, (n, oracle.rel_l2(y, want))


def test_fastconv_matches_reference_library(oracle, golden_ref):
    x, rep = golden_ref["fc_in"], golden_ref["fc_rep"]
    y = Fastconv(rep, x.shape[0])(x)
    assert oracle.error_db(golden_ref["fc_phased"], y) < -100
    assert oracle.error_db(golden_ref["fc_fused"], y) < -100
    assert oracle.rel_l2(y, oracle.fastconv(x, rep)) <= RTOL


def test_fastconv_shift_kernel(oracle, golden_ref):
    # tests/fastconv.cpp:341-366 (fused_v_multi, 64 samples, shift 2, scale 2)
    x, rep, shift = golden_ref["shift_in"], golden_ref["shift_rep"], 2
    y = Fastconv(rep, x.shape[0])(x)
    n = x.shape[1]
    assert oracle.error_db(2 * x[:, : n - shift], y[:, shift:]) < -100
    assert oracle.error_db(golden_ref["shift_fused"], y) < -100


def test_fastconv_matrix_of_coefficients(oracle, golden_ref):
    x, w = golden_ref["mat_in"], golden_ref["mat_rep"]
    y = Fastconv(w, x.shape[0])(x)
    assert oracle.error_db(golden_ref["mat_fused"], y) < -100
    assert oracle.rel_l2(y, oracle.fastconv(x, w)) <= RTOL


@pytest.mark.parametrize("n", [2048, 32768])
def test_replica_time_domain_fp64_on_gpu(oracle, n):
    torch = _torch()
    chirp = oracle.lfm_chirp(n, 100.0, n)
    want = np.conj(np.fft.fft(chirp))
    got = replica_spectrum(torch.from_numpy(chirp.astype(np.complex64)).cuda(), matched=True).cpu().numpy()
    # FP64 transform of the float-rounded chirp, then one rounding to complex64
    want32 = np.conj(np.fft.fft(chirp.astype(np.complex64).astype(np.complex128)))
    assert oracle.rel_l2(got, want32) < 1e-7
    assert oracle.rel_l2(got, want) < 2e-7
    rng = np.random.default_rng(n)
    x = crandn(rng, (8, n))
    y = Fastconv(chirp.astype(np.complex64), 8, kind="matched")(x)
    assert oracle.rel_l2(y, oracle.fastconv(x, want32.astype(np.complex64))) <= RTOL


def test_phased_equals_fused(oracle):
    # benchmarks/fastconv.cpp Impl1op (Fftm -> vmmul -> Fftm) vs Impl4vc (fused)
    torch = _torch()
    rows, n = 64, 8192
    rng = np.random.default_rng(11)
    x = crandn(rng, (rows, n))
    rep = crandn(rng, (n,))
    dx = torch.from_numpy(x).cuda()
    drep = torch.from_numpy(rep).cuda()
    tmp = Fftm(rows, n, fft_fwd, 1.0)(dx)
    tmp = vmmul(drep, tmp)
    y1 = Fftm(rows, n, fft_inv, 1.0 / n)(tmp)
    y2 = Fastconv(rep, rows)(dx)
    torch.cuda.synchronize()
    want = oracle.fastconv(x, rep)
    assert oracle.rel_l2(y1.cpu().numpy(), want) <= RTOL
    assert oracle.rel_l2(y2.cpu().numpy(), want) <= RTOL
    v = vmmul(drep, dx).cpu().numpy()
    np.testing.assert_allclose(v, rep[None, :] * x, rtol=1e-6, atol=1e-6)


def test_fastconv_inplace_strided_and_fewer_rows(oracle):
    torch = _torch()
    n, rows = 16384, 12
    rng = np.random.default_rng(3)
    big = crandn(rng, (rows, n + 32))
    x = big[:, :n]
    rep = crandn(rng, (n,))
    fc = Fastconv(rep, 32)
    y = fc(x)
    assert oracle.rel_l2(y, oracle.fastconv(x, rep)) <= RTOL
    dbig = torch.from_numpy(big).cuda()
    fc.in_place(dbig[:, :n])
    torch.cuda.synchronize()
    got = dbig.cpu().numpy()
    np.testing.assert_array_equal(got[:, :n], y)
    np.testing.assert_array_equal(got[:, n:], big[:, n:])  # padding untouched


def test_fastconv_full_size_pulse_compression(oracle):
    # 1024 pulses x 16384 samples, 8 echoes per pulse, LFM TBP 500 (full size)
    torch = _torch()
    job = synth.large_fastconv(seed=1)
    x, rep = job["data"], job["replica_spectrum"]
    dx = torch.from_numpy(x).cuda()
    fc = Fastconv(rep, x.shape[0])
    y = fc(dx).cpu().numpy()
    want = oracle.fastconv(x, rep)
    per_row = np.linalg.norm(y - want, axis=1) / np.linalg.norm(want, axis=1)
    assert per_row.max() <= RTOL, per_row.max()
    # linearity: f(a x1 + b x2) = a f(x1) + b f(x2)
    a, b = np.complex64(0.5 - 0.25j), np.complex64(-1.5)
    x2 = np.roll(x, 7, axis=1)
    y2 = fc(torch.from_numpy(x2).cuda()).cpu().numpy()
    y3 = fc(torch.from_numpy((a * x + b * x2).astype(np.complex64)).cuda()).cpu().numpy()
    assert oracle.rel_l2(y3, a * y.astype(np.complex128) + b * y2) <= 4 * RTOL
    # every echo compresses to a peak of about a * N at its delay
    n = x.shape[1]
    for p in range(4):
        for d, amp in zip(job["delays"][p], job["amplitudes"][p]):
            assert abs(y[p, int(d)]) > 0.5 * amp * n


@pytest.mark.parametrize("case", ["C1", "C2"])
def test_fastconv_accuracy_vs_fp32_cpu(oracle, case):
    """The fused fast convolution's error is no worse than 2x the FP32 CPU
    FFT's on the same seeded inputs: scipy's pocketfft complex64 stands in for
    the reference's FFTW3 FP32 path, which is not installed.  C1: 64 pulses x
    2048 samples, TBP 100; C2: 1024 pulses x 16384 samples with 8 echoes per
    pulse, TBP 500.  Both with the spectrum given and with the time-domain
    chirp transformed by the library in FP64 on the GPU."""
    import scipy.fft
    torch = _torch()
    job = synth.cpu_case(seed=0) if case == "C1" else synth.large_fastconv(seed=1)
    x, chirp = job["data"], job["chirp"].astype(np.complex64)
    spec = np.conj(np.fft.fft(chirp.astype(np.complex128))).astype(np.complex64)
    want = oracle.fastconv(x, spec)
    cpu = scipy.fft.ifft(scipy.fft.fft(x, axis=1) * spec, axis=1)
    assert cpu.dtype == np.complex64
    cpu_err = oracle.rel_l2(cpu, want)
    dx = torch.from_numpy(x).cuda()
    for fc in (Fastconv(spec, x.shape[0]), Fastconv(chirp, x.shape[0], kind="matched")):
        y = fc(dx).cpu().numpy()
        err = oracle.rel_l2(y, want)
        assert err <= RTOL and err <= 2 * cpu_err, (err, cpu_err)


def test_calls_follow_the_current_torch_stream(oracle):
    # a plan binds the current torch stream only when it changes: calls made
    # alternately under two streams, each on an input produced on its stream
    # behind a long kernel (a call queued on another stream would read that
    # input before it is written), must all equal the FP64 result
    import torch
    rng = np.random.default_rng(31)
    rows, n = 64, 4096
    rep = crandn(rng, (n,))
    x = torch.from_numpy(crandn(rng, (rows, n))).cuda()
    want = oracle.fastconv(x.cpu().numpy(), rep)
    fc = Fastconv(rep, rows)
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    outs = []
    for k in range(6):
        s = streams[k % 2]
        with torch.cuda.stream(s):
            torch.cuda._sleep(2_000_000)  # keeps the stream busy for about a millisecond
            xk = x * 1  # written on s after the sleep
            y = torch.empty_like(x)
            fc(xk, y)
            w = torch.empty_like(x)
            vmmul(torch.ones(n, dtype=torch.complex64, device="cuda"), y, w)
            outs.append((s, y, w))
    for s, y, w in outs:
        s.synchronize()
        assert oracle.rel_l2(y.cpu().numpy(), want) <= 2e-6
        np.testing.assert_array_equal(w.cpu().numpy(), y.cpu().numpy())
