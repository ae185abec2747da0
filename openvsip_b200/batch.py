"""Batched fast convolution: uneven jobs in one persistent, graph-replayed launch.

    b = Batch()                                  # tuned variant
    rid = b.add_replica(chirp, kind="matched")   # resident replica spectrum
    b.set_jobs([(x1, y1, rid), (x2, y2, rid2)])  # CUDA complex64 tensors, rows x n
    b.run(); b.sync()

Each job is one reference-style fast convolution
inv_fftm(vmmul<0>(R, fwd_fftm(x))) with scale 1/n (benchmarks/fastconv.cpp:
100-106); all jobs of a set run in one persistent kernel launch from a CUDA
graph (C ABI: fcb_batch_* in include/fcb200.h).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FcbJob, check, lib

_KINDS = {"spectrum": _lib.FCB_REPLICA_SPECTRUM, "time": _lib.FCB_REPLICA_TIME,
          "matched": _lib.FCB_REPLICA_TIME_MATCHED}


class Batch:
    """A set of fast-convolution jobs run together on the GPU."""

    def __init__(self, threads: int = 0):
        h = ctypes.c_void_p()
        check(lib().fcb_batch_create(int(threads), ctypes.byref(h)))
        self._h = h
        self._jobs = []  # keep tensors alive while the job table points at them

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h is not None:
            try:
                lib().fcb_batch_destroy(h)
            except Exception:
                pass

    def add_replica(self, replica, kind: str = "spectrum") -> int:
        """Make a replica resident; numpy (host) or CUDA tensor (device), complex64."""
        rid = ctypes.c_int()
        if type(replica).__module__.startswith("torch"):
            r = replica.contiguous().reshape(-1)
            check(lib().fcb_batch_add_replica(self._h, ctypes.c_void_p(r.data_ptr()), r.numel(), _KINDS[kind],
                                              _lib.FCB_DEVICE, ctypes.byref(rid)))
        else:
            r = np.ascontiguousarray(replica, dtype=np.complex64).reshape(-1)
            check(lib().fcb_batch_add_replica(self._h, ctypes.c_void_p(r.ctypes.data), r.size, _KINDS[kind],
                                              _lib.FCB_HOST, ctypes.byref(rid)))
        return rid.value

    def set_jobs(self, jobs, order: str = "longest_first", direct: bool = False) -> None:
        """jobs: iterable of (input, output, replica_id) with CUDA complex64
        tensors of shape (pulses, n); output may be the input (in place).
        direct=True launches without capturing a CUDA graph (for job sets that
        change with every run)."""
        arr = (FcbJob * max(1, len(jobs)))()
        keep = []
        for i, (x, y, rid) in enumerate(jobs):
            for t in (x, y):
                if not (type(t).__module__.startswith("torch") and t.is_cuda and t.dim() == 2 and t.stride(1) == 1):
                    raise TypeError("batch jobs take 2-D CUDA complex64 tensors with unit-stride rows")
            arr[i].in_ = x.data_ptr()
            arr[i].in_rs = x.stride(0) if x.shape[0] > 1 else x.shape[1]
            arr[i].out = y.data_ptr()
            arr[i].out_rs = y.stride(0) if y.shape[0] > 1 else y.shape[1]
            arr[i].pulses = x.shape[0]
            arr[i].n = x.shape[1]
            arr[i].replica = int(rid)
            keep.append((x, y))
        flags = (0 if order == "longest_first" else 1) | (2 if direct else 0)
        check(lib().fcb_batch_set_jobs(self._h, ctypes.cast(arr, ctypes.c_void_p), len(jobs), flags))
        self._jobs = keep

    def set_stream(self, stream) -> None:
        check(lib().fcb_batch_set_stream(self._h, ctypes.c_void_p(stream)))

    def run(self) -> None:
        """One graph launch: every job once (asynchronous on the batch stream)."""
        check(lib().fcb_batch_run(self._h))

    def sync(self) -> None:
        check(lib().fcb_batch_sync(self._h))

    def info(self) -> dict:
        u, s, g, t = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
        check(lib().fcb_batch_info(self._h, ctypes.byref(u), ctypes.byref(s), ctypes.byref(g), ctypes.byref(t)))
        return {"units": u.value, "samples": s.value, "grid": g.value, "threads": t.value}
