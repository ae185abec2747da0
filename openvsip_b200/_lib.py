"""ctypes binding of libfcb200.so (the C ABI declared in include/fcb200.h).

The library must have been built (``python -m openvsip_b200.build``); loading
fails loudly otherwise.  There is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfcb200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "fcb200.h")

FCB_OK = 0
FCB_ERR_INVALID = 1
FCB_ERR_UNSUPPORTED = 2
FCB_ERR_CUDA = 3
FCB_ERR_NOMEM = 4
FCB_ERR_TIMEOUT = 5
FCB_ERR_NODEVICE = 6

FCB_HOST = 0
FCB_DEVICE = 1
FCB_FORWARD = -1
FCB_INVERSE = +1
FCB_REPLICA_SPECTRUM = 0
FCB_REPLICA_TIME = 1
FCB_REPLICA_TIME_MATCHED = 2

_STATUS_NAMES = {
    FCB_ERR_INVALID: "invalid argument",
    FCB_ERR_UNSUPPORTED: "unsupported",
    FCB_ERR_CUDA: "CUDA error",
    FCB_ERR_NOMEM: "out of memory",
    FCB_ERR_TIMEOUT: "timeout",
    FCB_ERR_NODEVICE: "no device",
}


class FcbError(RuntimeError):
    """Raised for a non-zero fcb200 status; .status holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"fcb200: {_STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None

c_ll = ctypes.c_longlong
c_vp = ctypes.c_void_p
c_int = ctypes.c_int
c_float = ctypes.c_float

# (name, restype, argtypes) for every entry point in include/fcb200.h
SIGNATURES = {
    "fcb_last_error": (ctypes.c_char_p, []),
    "fcb_version": (ctypes.c_char_p, []),
    "fcb_init": (c_int, [c_int]),
    "fcb_supported_length": (c_int, [c_ll]),
    "fcb_plan_fftm": (c_int, [c_ll, c_ll, c_int, c_float, ctypes.POINTER(c_vp)]),
    "fcb_plan_fastconv": (c_int, [c_ll, c_ll, c_vp, c_ll, c_ll, c_int, c_int, ctypes.POINTER(c_vp)]),
    "fcb_plan_fft2d": (c_int, [c_ll, c_ll, c_int, c_float, ctypes.POINTER(c_vp)]),
    "fcb_exec": (c_int, [c_vp, c_vp, c_ll, c_vp, c_ll, c_ll, c_int]),
    "fcb_exec_async": (c_int, [c_vp, c_vp, c_ll, c_vp, c_ll, c_ll, c_int]),
    "fcb_supported_real_length": (c_int, [c_ll]),
    "fcb_plan_fftm_real": (c_int, [c_ll, c_ll, c_int, c_float, ctypes.POINTER(c_vp)]),
    "fcb_exec_r2c": (c_int, [c_vp, c_vp, c_ll, c_vp, c_ll, c_ll, c_int]),
    "fcb_exec_c2r": (c_int, [c_vp, c_vp, c_ll, c_vp, c_ll, c_ll, c_int]),
    "fcb_set_stream": (c_int, [c_vp, c_vp]),
    "fcb_sync": (c_int, [c_vp]),
    "fcb_destroy": (c_int, [c_vp]),
    "fcb_plan_info": (c_int, [c_vp, ctypes.POINTER(c_ll), ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                              ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "fcb_tune_set": (c_int, [c_ll, c_int, c_int]),
    "fcb_tune_get": (c_int, [c_ll, c_int]),
    "fcb_vmmul_rows": (c_int, [c_vp, c_vp, c_ll, c_vp, c_ll, c_ll, c_ll, c_vp]),
    "fcb_replica_spectrum": (c_int, [c_vp, c_ll, c_int, c_vp]),
    "fcb_replica_spectrum_noalloc": (c_int, [c_vp, c_ll, c_int, c_vp, c_vp]),
    "fcb_batch_create": (c_int, [c_int, ctypes.POINTER(c_vp)]),
    "fcb_batch_add_replica": (c_int, [c_vp, c_vp, c_ll, c_int, c_int, ctypes.POINTER(c_int)]),
    "fcb_batch_set_jobs": (c_int, [c_vp, c_vp, c_int, c_int]),
    "fcb_batch_run": (c_int, [c_vp]),
    "fcb_batch_set_stream": (c_int, [c_vp, c_vp]),
    "fcb_batch_sync": (c_int, [c_vp]),
    "fcb_batch_info": (c_int, [c_vp, ctypes.POINTER(c_ll), ctypes.POINTER(c_ll), ctypes.POINTER(c_int),
                               ctypes.POINTER(c_int)]),
    "fcb_batch_destroy": (c_int, [c_vp]),
}


class FcbJob(ctypes.Structure):
    """fcb_job (include/fcb200.h)."""
    _fields_ = [("in_", c_vp), ("in_rs", c_ll), ("out", c_vp), ("out_rs", c_ll), ("pulses", c_ll),
                ("n", c_ll), ("replica", c_int)]


def header_symbols() -> list[str]:
    """Names of the functions declared in include/fcb200.h."""
    text = open(HEADER).read()
    return re.findall(r"^FCB_API\s+[^(]*?\b(fcb_\w+)\s*\(", text, flags=re.M)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FcbError(FCB_ERR_NODEVICE,
                           f"{LIB_PATH} is missing: build it with `python -m openvsip_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            if hasattr(L, name):
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    msg = lib().fcb_last_error()
    return msg.decode() if msg else ""


def check(status: int) -> None:
    if status != FCB_OK:
        raise FcbError(status, last_error())
