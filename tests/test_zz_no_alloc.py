"""The no-allocation replica-spectrum entry point.

fcb_replica_spectrum_noalloc serves callers that must not allocate device
memory while they run (a real-time pulse-compression loop with a fixed memory
budget, or a process that reserves all device memory up front).  It keeps its
FP64 work buffers in an array built into the library instead of allocating
them per call, so it accepts powers of two up to 65536 samples.  Its results
are checked against numpy's FP64 FFT directly and against the allocating entry
point fcb_replica_spectrum, call after call, because the shared array keeps the
previous call's contents.

This file is collected last on purpose, so that a run that stops at the first
failure has already run every other test; it also passes on its own.
"""
import ctypes

import numpy as np
import pytest

from openvsip_b200 import _lib

pytestmark = pytest.mark.gpu
RTOL = 2e-6  # the relative-L2 tolerance used throughout the GPU tests


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _chirp(n, tbp, seed):
    rng = np.random.default_rng(seed)
    k = np.arange(n) / n - 0.5
    c = np.exp(1j * np.pi * tbp * k * k) + 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    return c.astype(np.complex64)


def _fp64_spectrum(x, matched):
    s = np.fft.fft(x.astype(np.complex128))
    return np.conj(s) if matched else s


def _rel(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n", [1, 2048, 65536])
def test_noalloc_spectrum_matches_fp64_and_allocating_entry_point(n):
    import torch
    L = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, (tbp, matched) in enumerate([(100.0, 1), (700.0, 0)]):  # two calls in a row
        host = _chirp(n, tbp, seed=call)
        x = torch.from_numpy(host).cuda()
        got = torch.full_like(x, float("nan"))
        _lib.check(L.fcb_replica_spectrum_noalloc(_ptr(x), n, matched, _ptr(got), stream))
        torch.cuda.synchronize()
        g = got.cpu().numpy()
        assert np.all(np.isfinite(g))
        assert _rel(g, _fp64_spectrum(host, matched)) <= RTOL, f"call {call} vs FP64"
        want = torch.empty_like(x)
        _lib.check(L.fcb_replica_spectrum(_ptr(x), n, matched, _ptr(want)))
        assert _rel(g, want.cpu().numpy()) <= RTOL, f"call {call} vs fcb_replica_spectrum"


def test_noalloc_in_place_on_its_own_stream():
    """In place (the kernel reads the whole input before it writes), issued on
    a stream other than the current one."""
    import torch
    L = _lib.lib()
    n = 4096
    host = _chirp(n, 300.0, seed=7)
    side = torch.cuda.Stream()
    x = torch.from_numpy(host).cuda()
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        _lib.check(L.fcb_replica_spectrum_noalloc(_ptr(x), n, 1, _ptr(x), ctypes.c_void_p(side.cuda_stream)))
    side.synchronize()
    assert _rel(x.cpu().numpy(), _fp64_spectrum(host, True)) <= RTOL


@pytest.mark.parametrize("n, code", [(131072, "INVALID"), (100000, "INVALID"), (1000, "UNSUPPORTED"),
                                     (0, "UNSUPPORTED")])
def test_noalloc_rejections(n, code):
    import torch
    L = _lib.lib()
    x = torch.zeros(16, dtype=torch.complex64, device="cuda")
    rc = L.fcb_replica_spectrum_noalloc(_ptr(x), n, 1, _ptr(x), None)
    assert rc == getattr(_lib, "FCB_ERR_" + code)
    if code == "INVALID":
        assert "65536" in _lib.last_error()
    else:
        assert "power of two" in _lib.last_error()
