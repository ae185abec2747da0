import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100) device")
    config.addinivalue_line("markers", "slow: long-running")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _cuda_available()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden_fft_ext():
    return dict(np.load(os.path.join(GOLDEN, "fft_ext_cc.npz")))


@pytest.fixture(scope="session")
def golden_ref():
    return dict(np.load(os.path.join(GOLDEN, "ref_outputs.npz")))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.lib()
    return o


def crandn(rng, shape, scale=1.0):
    return ((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * scale).astype(np.complex64)


class pinned_variant:
    """Temporarily select a kernel variant (fcb_tune_set) for length n and kind
    (0 forward, 1 inverse, 2 fused), restoring the previous one on exit."""

    def __init__(self, n, kind, threads):
        self.n, self.kind, self.threads = n, kind, threads

    def __enter__(self):
        from openvsip_b200 import _lib
        self.lib = _lib.lib()
        self.saved = self.lib.fcb_tune_get(self.n, self.kind)
        _lib.check(self.lib.fcb_tune_set(self.n, self.kind, self.threads))
        return self

    def __exit__(self, *exc):
        from openvsip_b200 import _lib
        _lib.check(self.lib.fcb_tune_set(self.n, self.kind, self.saved))
