"""Host-side mirror of the reference's fast-convolution API on the fcb200 backend.

Names and argument meanings follow the reference:

* ``Fftm(rows, cols, direction, scale)`` -- ``vsip::Fftm<complex<float>,
  complex<float>, row, D, by_reference>`` (src/vsip/impl/signal/fft.hpp:134-161,
  src/ovxx/signal/fft.hpp:374-436): construct once per domain and scale, then
  ``fftm(in, out)`` (out of place) or ``fftm(inout)`` (in place); calls may pass
  fewer rows than planned.
* ``vmmul(v, m)`` -- ``vsip::vmmul<0>`` (src/vsip/impl/vmmul.hpp:114-128):
  ``out[r][c] = v[c] * m[r][c]``.
* ``Fastconv(weights, rows)`` -- the fused expression
  ``inv_fftm(vmmul<0>(weights, for_fftm(in)))`` with the inverse scaled by 1/N
  (tests/fastconv.cpp:188-211; benchmarks/fastconv.cpp:100-106).  A weight
  matrix gives ``inv_fftm(weights * for_fftm(in))`` (tests/fastconv.cpp:213-246).

Arrays are numpy ``complex64`` (host memory, copied through the GPU inside the
call) or torch ``complex64`` CUDA tensors (device memory; asynchronous on the
current torch stream).  Rows must be unit-stride.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FcbError, check, lib

fft_fwd = -2  # reference tag values (src/ovxx/signal/fft/backend.hpp:20-22)
fft_inv = -1


def _exponent(direction: int) -> int:
    """Map the reference's direction tag to the transform exponent.  Only the
    tags are accepted: fft_inv (-1) and the forward exponent (-1) share a value."""
    if direction == fft_fwd:
        return _lib.FCB_FORWARD
    if direction == fft_inv:
        return _lib.FCB_INVERSE
    raise ValueError(f"direction must be fft_fwd ({fft_fwd}) or fft_inv ({fft_inv}), got {direction}")


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


_torch = None
_raw_stream = None  # (torch's current-device query, its raw current-stream query), or ()


def _torch_mod():
    global _torch
    if _torch is None:
        import torch
        _torch = torch
    return _torch


def _stream_handle() -> int:
    """Raw handle of the current torch stream on the current device.  The public
    torch.cuda.current_stream() builds a Stream object on every call (about
    3 us, a quarter of a small call's host time); torch's raw accessors answer
    the same in under 0.1 us and are used where this torch has them."""
    global _raw_stream
    t = _torch_mod()
    if _raw_stream is None:
        dev = getattr(t._C, "_cuda_getDevice", None)
        raw = getattr(t._C, "_cuda_getCurrentRawStream", None)
        _raw_stream = (dev, raw) if dev is not None and raw is not None else ()
    if _raw_stream:
        return _raw_stream[1](_raw_stream[0]())
    return t.cuda.current_stream().cuda_stream


def _desc(x, writable: bool, real: bool = False):
    """(pointer, rows, cols, row_stride, where) of a 2-D complex64 (or, with
    real=True, float32) array/tensor; the stride counts elements."""
    el = 4 if real else 8
    if type(x) is not np.ndarray and _is_torch(x):
        t = _torch_mod()
        if x.dtype is not (t.float32 if real else t.complex64):
            raise TypeError("expected a float32 tensor" if real else "expected a complex64 tensor")
        if not x.is_cuda:
            raise TypeError("torch tensors must be on a CUDA device; use numpy arrays for host data")
        shape = x.shape
        if len(shape) == 1:  # one row
            if x.stride(0) != 1:
                raise ValueError("expected a 2-D tensor with unit-stride rows")
            return x.data_ptr(), 1, shape[0], shape[0], _lib.FCB_DEVICE
        st = x.stride()
        if len(shape) != 2 or st[1] != 1:
            raise ValueError("expected a 2-D tensor with unit-stride rows")
        rows, cols = shape
        return x.data_ptr(), rows, cols, st[0] if rows > 1 else cols, _lib.FCB_DEVICE
    a = x
    if not isinstance(a, np.ndarray) or a.dtype != (np.float32 if real else np.complex64):
        raise TypeError("expected a numpy float32 array" if real else "expected a numpy complex64 array")
    if a.ndim == 1:
        a = a.reshape(1, -1)
    if a.ndim == 2 and a.size == 0:  # empty: numpy reports zero strides, nothing is accessed
        return a.ctypes.data, a.shape[0], a.shape[1], max(1, a.shape[1]), _lib.FCB_HOST
    if a.ndim != 2 or (a.shape[1] > 1 and a.strides[1] != el) or a.strides[0] % el:
        raise ValueError("expected a 2-D array with unit-stride rows")
    if writable and not a.flags.writeable:
        raise ValueError("output array is read-only")
    rs = a.strides[0] // el if a.shape[0] > 1 else a.shape[1]  # one row: any stride is fine
    return a.ctypes.data, a.shape[0], a.shape[1], rs, _lib.FCB_HOST




def _empty_like(x):
    if _is_torch(x):
        import torch
        return torch.empty_like(x, memory_format=torch.contiguous_format)
    return np.empty(x.shape, dtype=np.complex64)


def _empty(like, shape, real: bool):
    """New array (numpy) or CUDA tensor on like's device, float32 or complex64."""
    if _is_torch(like):
        import torch
        return torch.empty(shape, dtype=torch.float32 if real else torch.complex64, device=like.device)
    return np.empty(shape, dtype=np.float32 if real else np.complex64)


def _transposed(x):
    """Contiguous transpose: the column-major copy the reference's DDA layer makes
    for a column-axis Fftm (query_layout asks for tuple<1,0,2>)."""
    if _is_torch(x):
        return x.t().contiguous()
    return np.ascontiguousarray(x.T)


def _put_transposed(out, yt):
    if _is_torch(out):
        out.copy_(yt.t())
    else:
        out[...] = yt.T
    return out


class _Plan:
    _handle = None
    _stream = None  # the stream handle last bound to the plan (fcb_set_stream)

    def _bind_stream(self, where) -> None:
        """Device calls run on the current torch stream; the plan is told only
        when that stream changes."""
        if where == _lib.FCB_DEVICE:
            s = _stream_handle()
            if s != self._stream:
                check(lib().fcb_set_stream(self._handle, ctypes.c_void_p(s)))
                self._stream = s

    def __del__(self):
        h, self._handle = self._handle, None
        if h is not None and lib is not None:
            try:
                lib().fcb_destroy(h)
            except Exception:
                pass

    def info(self) -> dict:
        n = ctypes.c_longlong()
        cl = ctypes.c_int()
        rpc = ctypes.c_int()
        sm = ctypes.c_int()
        th = ctypes.c_int()
        check(lib().fcb_plan_info(self._handle, ctypes.byref(n), ctypes.byref(cl), ctypes.byref(rpc),
                                  ctypes.byref(sm), ctypes.byref(th)))
        return {"n": n.value, "cluster_ctas": cl.value, "rows_per_cta": rpc.value, "smem_bytes": sm.value,
                "threads": th.value}

    def _exec(self, inp, out, wait: bool = True):
        ip, r, c, irs, iw = _desc(inp, False)
        op, r2, c2, ors, ow = _desc(out, True)
        if (r, c) != (r2, c2):
            raise ValueError(f"shape mismatch {(r, c)} vs {(r2, c2)}")
        n = getattr(self, "_n", self.cols)  # transform length (Fftm along columns: rows)
        if c != n:
            raise ValueError(f"row length {c} != planned {n}")
        if iw != ow:
            raise ValueError("input and output must both be host arrays or both device tensors")
        self._bind_stream(iw)
        fn = lib().fcb_exec if wait else lib().fcb_exec_async
        check(fn(self._handle, ctypes.c_void_p(ip), irs, ctypes.c_void_p(op), ors, r, iw))
        return out

    def submit(self, inp, out):
        """Queue ``plan(inp, out)`` and return at once (fcb_exec_async).  With
        host arrays the copies in, the kernels and the copies out run in the
        background, and calls submitted back to back overlap on the PCIe link;
        both arrays (pinned host memory, e.g. from torch's pin_memory) must stay
        untouched until sync().  With CUDA tensors it is the same as a call."""
        return self._exec(inp, out, wait=False)

    def sync(self) -> None:
        """Wait for everything submitted to this plan."""
        check(lib().fcb_sync(self._handle))

    def __call__(self, inp, out=None):
        """``plan(in, out)`` by reference, ``plan(inout)`` ... see subclasses."""
        raise NotImplementedError


row = 0  # axis tags, values of vsip::row / vsip::col (src/vsip/support.hpp:167-168):
col = 1  # Fftm<I, O, row, ...> transforms each row, Fftm<I, O, col, ...> each column


class Fftm(_Plan):
    """Multiple FFT on the GPU (vsip::Fftm<C, C, A, D, R>).

    axis=row (default) transforms each of the `rows` rows of length `cols`;
    axis=col transforms each of the `cols` columns of length `rows`.  Column
    data is transposed into contiguous rows and back around the row kernel, as
    the reference's DDA layer does for its FFTW backend."""

    def __init__(self, rows: int, cols: int, direction: int = fft_fwd, scale: float = 1.0, axis: int = row):
        self.rows, self.cols = int(rows), int(cols)
        self.axis = _axis(axis)
        self.exponent = _exponent(direction)
        self.scale = float(scale)
        n, count = (self.cols, self.rows) if self.axis == row else (self.rows, self.cols)
        h = ctypes.c_void_p()
        check(lib().fcb_plan_fftm(n, count, self.exponent, self.scale, ctypes.byref(h)))
        self._handle = h
        self._n = n

    def __call__(self, inp, out=None):
        """By reference: ``fftm(in, out)``; ``fftm(in)`` returns a new result (by value)."""
        if out is None:
            out = _empty_like(inp)
        if self.axis == col:
            return _put_transposed(out, self._rows(_transposed(inp)))
        return self._exec(inp, out)

    def in_place(self, inout):
        if self.axis == col:
            return _put_transposed(inout, self._rows(_transposed(inout)))
        return self._exec(inout, inout)

    def _rows(self, xt):
        return self._exec(xt, _empty_like(xt))


def _axis(axis: int) -> int:
    if axis not in (row, col):
        raise ValueError("axis must be row (0) or col (1)")
    return axis


class FftmReal(_Plan):
    """Real-input multiple FFT on the GPU.

    direction fft_fwd: vsip::Fftm<float, complex<float>, A, fft_fwd> -- real
    input of `rows` x `cols`, complex output with n/2 + 1 bins along the axis.
    direction fft_inv: vsip::Fftm<complex<float>, float, A, fft_inv> -- the
    half spectrum in, real output of `rows` x `cols` (unnormalised; pass
    scale=1/n for the inverse of the forward).  rows x cols is always the real
    side's domain, as in the reference; axis as for Fftm."""

    def __init__(self, rows: int, cols: int, direction: int = fft_fwd, scale: float = 1.0, axis: int = row):
        self.rows, self.cols = int(rows), int(cols)
        self.axis = _axis(axis)
        self.exponent = _exponent(direction)
        self.scale = float(scale)
        self.n, self.count = (self.cols, self.rows) if self.axis == row else (self.rows, self.cols)
        self.bins = self.n // 2 + 1
        h = ctypes.c_void_p()
        check(lib().fcb_plan_fftm_real(self.n, self.count, self.exponent, self.scale, ctypes.byref(h)))
        self._handle = h

    def output_shape(self):
        if self.exponent == _lib.FCB_INVERSE:
            return (self.rows, self.cols)
        return (self.count, self.bins) if self.axis == row else (self.bins, self.count)

    def __call__(self, inp, out=None):
        fwd = self.exponent == _lib.FCB_FORWARD
        if out is None:
            out = _empty(inp, self.output_shape(), real=not fwd)
        if self.axis == col:
            yt = _empty(inp, (self.count, self.n if not fwd else self.bins), real=not fwd)
            self._rows(_transposed(inp), yt)
            return _put_transposed(out, yt)
        return self._rows(inp, out)

    def _rows(self, inp, out):
        fwd = self.exponent == _lib.FCB_FORWARD
        ip, r, c, irs, iw = _desc(inp, False, real=fwd)
        op, r2, c2, ors, ow = _desc(out, True, real=not fwd)
        want_in, want_out = (self.n, self.bins) if fwd else (self.bins, self.n)
        if c != want_in or c2 != want_out or r != r2:
            raise ValueError(f"shapes {(r, c)} -> {(r2, c2)} do not match n={self.n}")
        if iw != ow:
            raise ValueError("input and output must both be host arrays or both device tensors")
        self._bind_stream(iw)
        fn = lib().fcb_exec_r2c if fwd else lib().fcb_exec_c2r
        check(fn(self._handle, ctypes.c_void_p(ip), irs, ctypes.c_void_p(op), ors, r, iw))
        return out


class Fft2d(_Plan):
    """2-D FFT of a rows x cols matrix on the GPU (vsip::Fft<const_Matrix, C, C,
    D>, src/vsip/impl/signal/fft.hpp:75-132): rows, then columns, output times
    scale.  Dimensions: any supported row length (powers of two in [64, 16384]
    take the two-pass transposing path, other sizes two row passes and two
    transposes)."""

    def __init__(self, rows: int, cols: int, direction: int = fft_fwd, scale: float = 1.0):
        self.rows, self.cols = int(rows), int(cols)
        self.exponent = _exponent(direction)
        self.scale = float(scale)
        h = ctypes.c_void_p()
        check(lib().fcb_plan_fft2d(self.rows, self.cols, self.exponent, self.scale, ctypes.byref(h)))
        self._handle = h

    def __call__(self, inp, out=None):
        if out is None:
            out = _empty_like(inp)
        return self._exec(inp, out)


class Fastconv(_Plan):
    """Fused fast convolution: ``inv_fftm(vmmul<0>(weights, for_fftm(in)))``.

    weights: a replica spectrum vector (kind="spectrum", the vmmul vector of the
    reference), or a time-domain replica transformed on the GPU in FP64
    (kind="time": FFT(w); kind="matched": conj(FFT(w))).  A 2-D weights array
    with one row per data row is the matrix-of-coefficients form."""

    _KINDS = {"spectrum": _lib.FCB_REPLICA_SPECTRUM, "time": _lib.FCB_REPLICA_TIME,
              "matched": _lib.FCB_REPLICA_TIME_MATCHED}

    def __init__(self, weights, rows: int, kind: str = "spectrum"):
        if kind not in self._KINDS:
            raise ValueError(f"kind must be one of {sorted(self._KINDS)}")
        if not _is_torch(weights):
            weights = np.ascontiguousarray(weights, dtype=np.complex64)
        wp, wr, wc, wrs, ww = _desc(weights, False)
        self.rows, self.cols = int(rows), int(wc)
        self.replica_rows = wr
        h = ctypes.c_void_p()
        check(lib().fcb_plan_fastconv(self.cols, self.rows, ctypes.c_void_p(wp), wr, wrs,
                                      self._KINDS[kind], ww, ctypes.byref(h)))
        self._handle = h

    def __call__(self, inp, out=None):
        if out is None:
            out = _empty_like(inp)
        return self._exec(inp, out)

    def in_place(self, inout):
        return self._exec(inout, inout)


def vmmul(v, m, out=None):
    """vmmul<0>(v, m): out[r][c] = v[c] * m[r][c], on the GPU.

    v and m must be CUDA complex64 tensors (device data); the op is queued on
    the current torch stream."""
    import torch
    if not (_is_torch(v) and _is_torch(m) and v.is_cuda and m.is_cuda):
        raise TypeError("vmmul runs on the GPU: pass CUDA complex64 tensors")
    if out is None:
        out = torch.empty_like(m)
    mp, r, c, mrs, _ = _desc(m, False)
    op, r2, c2, ors, _ = _desc(out, True)
    if not v.is_contiguous():
        v = v.contiguous()
    if v.numel() != c or (r2, c2) != (r, c):
        raise ValueError("shape mismatch")
    stream = _stream_handle()
    check(lib().fcb_vmmul_rows(ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(mp), mrs, ctypes.c_void_p(op),
                               ors, r, c, ctypes.c_void_p(stream)))
    return out


def replica_spectrum(replica, matched: bool = True):
    """FP64-on-GPU spectrum of a time-domain replica (CUDA complex64 tensor)."""
    import torch
    if not (_is_torch(replica) and replica.is_cuda):
        raise TypeError("pass a CUDA complex64 tensor")
    r = replica.contiguous().reshape(-1)
    out = torch.empty_like(r)
    torch.cuda.current_stream().synchronize()
    check(lib().fcb_replica_spectrum(ctypes.c_void_p(r.data_ptr()), r.numel(), int(bool(matched)),
                                     ctypes.c_void_p(out.data_ptr())))
    return out


def supported_length(n: int) -> bool:
    return bool(lib().fcb_supported_length(int(n)))


__all__ = ["Fftm", "FftmReal", "Fft2d", "Fastconv", "vmmul", "replica_spectrum", "supported_length", "fft_fwd",
           "fft_inv", "row", "col",
           "FcbError"]
