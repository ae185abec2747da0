"""C-ABI checks that need no GPU: the library loads, exports every entry point
declared in include/fcb200.h, and rejects bad arguments with the documented
status codes before touching a device."""
import ctypes
import subprocess

import numpy as np
import pytest

from conftest import HAS_GPU
from openvsip_b200 import _lib


def test_library_exports_every_header_symbol():
    names = _lib.header_symbols()
    assert len(names) >= 13
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in names if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    L = _lib.lib()
    for n in names:
        assert hasattr(L, n)


def test_every_export_is_declared():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    fcb = {n for n in exported if n.startswith("fcb_")}
    assert fcb <= set(_lib.header_symbols())


def test_supported_lengths():
    L = _lib.lib()
    # powers of two up to 65536 (one fused pass); any other length up to
    # 32768 (Bluestein through power-of-two work rows of at most 65536)
    for n in (1, 2, 3, 4, 18, 19, 68, 252, 768, 1024, 32767, 32768, 65536):
        assert L.fcb_supported_length(n) == 1
    for n in (0, 32769, 40000, 65535, 131072, -4):
        assert L.fcb_supported_length(n) == 0


def test_argument_errors_without_device():
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.fcb_plan_fftm(40000, 4, -1, 1.0, ctypes.byref(h)) == _lib.FCB_ERR_UNSUPPORTED
    assert b"power of two" in L.fcb_last_error()
    assert L.fcb_plan_fftm(1024, 4, 0, 1.0, ctypes.byref(h)) == _lib.FCB_ERR_INVALID
    assert L.fcb_plan_fftm(1024, 4, -1, 1.0, None) == _lib.FCB_ERR_INVALID
    assert L.fcb_exec(None, None, 0, None, 0, 1, 0) == _lib.FCB_ERR_INVALID
    assert L.fcb_plan_fastconv(1024, 4, None, 1, 1024, 0, 0, ctypes.byref(h)) == _lib.FCB_ERR_INVALID


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_no_device_is_reported():
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.fcb_plan_fftm(1024, 4, -1, 1.0, ctypes.byref(h)) == _lib.FCB_ERR_NODEVICE
    assert L.fcb_init(0) == _lib.FCB_ERR_NODEVICE
    with pytest.raises(_lib.FcbError):
        from openvsip_b200 import Fftm
        Fftm(4, 1024)


def test_python_api_validates_types():
    from openvsip_b200 import vsip as signal
    with pytest.raises(ValueError):
        signal._exponent(5)
    assert signal._exponent(signal.fft_fwd) == _lib.FCB_FORWARD
    assert signal._exponent(signal.fft_inv) == _lib.FCB_INVERSE
    with pytest.raises(TypeError):
        signal._desc(np.zeros((2, 4), dtype=np.complex128), False)
    with pytest.raises(ValueError):
        signal._desc(np.zeros((2, 4, 2), dtype=np.complex64), False)
    ptr, r, c, rs, where = signal._desc(np.zeros((3, 8), dtype=np.complex64)[:, :4], False)
    assert (r, c, rs, where) == (3, 4, 8, _lib.FCB_HOST)


def test_empty_arrays_are_described_without_strides():
    # numpy reports zero strides for empty arrays; an empty call must still pass
    import numpy as np
    from openvsip_b200.vsip import _desc
    assert _desc(np.zeros((0, 1024), dtype=np.complex64), False)[1:] == (0, 1024, 1024, 0)
    assert _desc(np.zeros((0, 16), dtype=np.float32), False, real=True)[1:] == (0, 16, 16, 0)


def test_python_api_rejects_unsuitable_tensors():
    # the tensor checks run before any library call: host (CPU) tensors, other
    # dtypes, more than two dimensions and non-unit-stride rows are refused
    import torch
    from openvsip_b200.vsip import _desc
    with pytest.raises(TypeError):
        _desc(torch.zeros(2, 4, dtype=torch.complex64), False)  # host tensor: use numpy for host data
    with pytest.raises(TypeError):
        _desc(torch.zeros(2, 4, dtype=torch.complex128), False)
    with pytest.raises(TypeError):
        _desc(torch.zeros(2, 4, dtype=torch.complex64), False, real=True)
