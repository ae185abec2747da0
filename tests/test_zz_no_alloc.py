"""The no-allocation replica-spectrum entry point.

fcb_replica_spectrum_noalloc serves callers that must not allocate device
memory while they run (a real-time pulse-compression loop with a fixed memory
budget, or a process that reserves all device memory up front).  It keeps its
FP64 work buffers in an array built into the library instead of allocating
them per call, so it accepts at most 65536 samples.  Its results must match the
allocating entry point fcb_replica_spectrum, call after call, because the
shared array keeps the previous call's contents.

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


@pytest.mark.parametrize("n", [2048, 65536])
def test_noalloc_spectrum_matches_allocating_entry_point(n):
    import torch
    L = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, (tbp, matched) in enumerate([(100.0, 1), (700.0, 0)]):  # two calls in a row
        x = torch.from_numpy(_chirp(n, tbp, seed=call)).cuda()
        want = torch.empty_like(x)
        _lib.check(L.fcb_replica_spectrum(_ptr(x), n, matched, _ptr(want)))
        got = torch.full_like(x, float("nan"))
        _lib.check(L.fcb_replica_spectrum_noalloc(_ptr(x), n, matched, _ptr(got), stream))
        torch.cuda.synchronize()
        w = want.cpu().numpy().astype(np.complex128)
        g = got.cpu().numpy().astype(np.complex128)
        assert np.all(np.isfinite(g))
        assert np.linalg.norm(g - w) / np.linalg.norm(w) <= RTOL, f"call {call}"


def test_noalloc_rejects_lengths_beyond_its_array():
    import torch
    L = _lib.lib()
    x = torch.zeros(16, dtype=torch.complex64, device="cuda")
    rc = L.fcb_replica_spectrum_noalloc(_ptr(x), 131072, 1, _ptr(x), None)
    assert rc == _lib.FCB_ERR_INVALID
    assert "65536" in _lib.last_error()
