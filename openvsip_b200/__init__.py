"""openvsip_b200 -- B200-native (sm_100a) fast-convolution backend for OpenVSIP.

The compute path is libfcb200.so (hand-written CUDA, C ABI in include/fcb200.h);
this package is its Python host binding: the reference-shaped API
(``Fftm``, ``vmmul``, ``Fastconv``), batched uneven jobs, the serving loop and
the synthetic workload generators.
"""
from ._lib import FcbError, lib  # noqa: F401
from . import synth  # noqa: F401
from .vsip import Fastconv, Fft2d, Fftm, fft_fwd, fft_inv, replica_spectrum, supported_length, vmmul  # noqa: F401

__version__ = "0.1.0"
