"""openvsip_b200 -- B200-native (sm_100a) fast-convolution backend for OpenVSIP.

The compute path is libfcb200.so (hand-written CUDA, C ABI in include/fcb200.h);
this package is its Python host binding: the reference-shaped API
(``Fftm``, ``vmmul``, ``Fastconv``), batched uneven jobs, the serving loop and
the synthetic workload generators.
"""
from ._lib import FcbError, lib  # noqa: F401
from . import synth  # noqa: F401
from .vsip import (Fastconv, Fft2d, Fftm, FftmReal, col, fft_fwd, fft_inv, replica_spectrum, row,  # noqa: F401
                   supported_length, vmmul)

__version__ = "0.1.0"
