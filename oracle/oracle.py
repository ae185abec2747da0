"""CPU oracle for the fast-convolution path -- TEST INFRASTRUCTURE ONLY.

Only the tests, the smoke check and the benchmark's CPU-baseline leg use this
module, and only as the checker; the product (``openvsip_b200``) never imports
it.

Two FP64 restatements of the reference's arithmetic are offered:

* ``liboracle.so`` (fcoracle.c): the reference's generic O(N^2) DFT
  (src/ovxx/signal/fft/dft.hpp:57-66), its row-wise Fftm loop (dft.hpp:1040-1058),
  vmmul<0> (src/ovxx/expr/vmmul.hpp:53-59), the 1/N scale pass
  (src/ovxx/signal/fft/workspace.hpp:474-478) and the test metric test::diff
  (support/test/diff.hpp:41-96), plus an FP64 radix-2 FFT.
* numpy's float64 FFT (pocketfft) for shapes where O(N^2) is too slow; it is
  cross-checked against the C DFT by the tests.

The fast-convolution definition followed here is the reference benchmark's
phased form (benchmarks/fastconv.cpp:100-106):
``inv_fftm(vmmul<0>(replica, for_fftm(data)))`` with scale 1/N on the inverse.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> None:
    """Compile liboracle.so (and, where the reference sources exist, _ref/)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        fp = ctypes.POINTER(ctypes.c_float)
        L.orc_dft_c64.argtypes = [dp, ctypes.c_long, dp, ctypes.c_long, ctypes.c_long,
                                  ctypes.c_int, ctypes.c_double]
        L.orc_fft_c64.argtypes = [dp, dp, ctypes.c_long, ctypes.c_int, ctypes.c_double]
        L.orc_fftm_rows_c64.argtypes = [dp, ctypes.c_long, dp, ctypes.c_long, ctypes.c_long,
                                        ctypes.c_long, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_vmmul_rows_c64.argtypes = [dp, dp, ctypes.c_long, dp, ctypes.c_long,
                                         ctypes.c_long, ctypes.c_long]
        L.orc_fastconv_c64.argtypes = [fp, ctypes.c_long, ctypes.c_long, fp, ctypes.c_long,
                                       dp, ctypes.c_int]
        L.orc_fastconv_c32.argtypes = [fp, ctypes.c_long, ctypes.c_long, fp, ctypes.c_long,
                                       fp, ctypes.c_int]
        L.orc_error_db.argtypes = [dp, dp, ctypes.c_long]
        L.orc_error_db.restype = ctypes.c_double
        L.orc_lfm_chirp_c64.argtypes = [ctypes.c_long, ctypes.c_double, ctypes.c_long, dp]
        _LIB = L
    return _LIB


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def dft_rows(x: np.ndarray, exponent: int, scale: float = 1.0, method: int = 0) -> np.ndarray:
    """Row-wise DFT in FP64 through the C oracle (method 0: O(N^2) DFT, 1: FFT)."""
    x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.complex128)
    rows, cols = x.shape
    out = np.empty_like(x)
    lib().orc_fftm_rows_c64(_dp(x), cols, _dp(out), cols, rows, cols, exponent, scale, method)
    return out


def fft_rows(x: np.ndarray, exponent: int, scale: float = 1.0) -> np.ndarray:
    """Row-wise FP64 FFT via numpy (pocketfft); exponent -1 forward, +1 inverse."""
    x = np.asarray(x, dtype=np.complex128)
    if exponent < 0:
        y = np.fft.fft(x, axis=-1)
    else:
        y = np.fft.ifft(x, axis=-1) * x.shape[-1]
    return y * scale


def vmmul_rows(v: np.ndarray, m: np.ndarray) -> np.ndarray:
    """vmmul<0>: out[r][c] = v[c] * m[r][c] (src/ovxx/expr/vmmul.hpp:53-59)."""
    return np.asarray(v, dtype=np.complex128)[None, :] * np.asarray(m, dtype=np.complex128)


def fastconv(x: np.ndarray, rep_spec: np.ndarray, method: str = "numpy") -> np.ndarray:
    """FP64 fast convolution of complex64 rows with a replica spectrum.

    rep_spec is one row (shared) or one row per input row (matrix of
    coefficients, tests/fastconv.cpp:213-246).  method "numpy" (pocketfft FP64),
    "fft" (C radix-2 FP64) or "dft" (C O(N^2) DFT, the reference's generic
    backend arithmetic)."""
    x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.complex64)
    rows, cols = x.shape
    rep = np.ascontiguousarray(rep_spec, dtype=np.complex64)
    if method == "numpy":
        f = fft_rows(x, -1)
        return fft_rows(f * rep.astype(np.complex128), +1, 1.0 / cols)
    rep_rs = cols if rep.ndim == 2 else 0
    out = np.empty((rows, cols), dtype=np.complex128)
    xf = x.view(np.float32)
    rf = rep.view(np.float32)
    lib().orc_fastconv_c64(_fp(xf), rows, cols, _fp(rf), rep_rs, _dp(out),
                           0 if method == "dft" else 1)
    return out


def fastconv_f32(x: np.ndarray, rep_spec: np.ndarray, threads: int = 0) -> np.ndarray:
    """FP32 radix-2 fast convolution on the CPU (speed baseline, not an oracle)."""
    x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.complex64)
    rows, cols = x.shape
    rep = np.ascontiguousarray(rep_spec, dtype=np.complex64)
    rep_rs = cols if rep.ndim == 2 else 0
    out = np.empty_like(x)
    lib().orc_fastconv_c32(_fp(x.view(np.float32)), rows, cols, _fp(rep.view(np.float32)),
                           rep_rs, _fp(out.view(np.float32)), threads)
    return out


def error_db(a: np.ndarray, b: np.ndarray) -> float:
    """Reference accuracy metric test::diff (support/test/diff.hpp:41-96)."""
    a = np.ascontiguousarray(a, dtype=np.complex128).ravel()
    b = np.ascontiguousarray(b, dtype=np.complex128).ravel()
    return float(lib().orc_error_db(_dp(a), _dp(b), a.size))


def rel_l2(y: np.ndarray, ref: np.ndarray) -> float:
    """||y - ref||_2 / ||ref||_2 computed in FP64."""
    y = np.asarray(y, dtype=np.complex128)
    ref = np.asarray(ref, dtype=np.complex128)
    return float(np.linalg.norm(y - ref) / np.linalg.norm(ref))


def lfm_chirp(length: int, tbp: float, n_out: int | None = None) -> np.ndarray:
    """LFM chirp exp(j pi tbp (n/L - 1/2)^2), n < L, zero-padded (FP64, C)."""
    n_out = length if n_out is None else n_out
    out = np.empty(n_out, dtype=np.complex128)
    lib().orc_lfm_chirp_c64(length, tbp, n_out, _dp(out))
    return out


def replica_spectrum(chirp: np.ndarray) -> np.ndarray:
    """Matched-filter replica spectrum conj(FFT(chirp)) in FP64."""
    return np.conj(np.fft.fft(np.asarray(chirp, dtype=np.complex128)))


REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")


def have_reference_build() -> bool:
    return os.path.exists(REF_DRIVER)
