"""Edge cases of the row kernels on the GPU: empty calls, a plan for zero rows,
single rows at odd strides, row counts that leave CTAs (or clusters) partly
empty, zero and negative scales, and calls that must be refused."""
import numpy as np
import pytest

from conftest import crandn
from openvsip_b200 import FcbError, Fastconv, Fftm, fft_fwd, fft_inv

pytestmark = pytest.mark.gpu
RTOL = 2e-6


def test_empty_calls_are_no_ops():
    import torch
    f = Fftm(4, 1024, fft_fwd, 1.0)
    out = f(np.zeros((0, 1024), dtype=np.complex64))
    assert out.shape == (0, 1024)
    fc = Fastconv(np.ones(1024, dtype=np.complex64), 4)
    d = torch.zeros(0, 1024, dtype=torch.complex64, device="cuda")
    assert fc(d).shape == (0, 1024)
    z = Fftm(0, 256, fft_fwd, 1.0)  # a plan for zero rows accepts only empty calls
    assert z(np.zeros((0, 256), dtype=np.complex64)).shape == (0, 256)
    with pytest.raises(FcbError):
        z(np.zeros((1, 256), dtype=np.complex64))


@pytest.mark.parametrize("n,rows", [(256, 1), (256, 17), (256, 33), (1024, 5), (4096, 3), (8192, 3),
                                    (32768, 3), (65536, 1), (1000, 7)])
def test_partial_tiles_and_single_rows(oracle, n, rows):
    # rows that leave the last CTA (several rows per CTA at short lengths) or
    # cluster partly empty; inactive rows must write nothing
    rng = np.random.default_rng(n + rows)
    x = crandn(rng, (rows, n))
    rep = crandn(rng, (n,))
    guard = crandn(rng, (rows + 2, n))
    out = guard.copy()
    Fastconv(rep, rows)(x, out[1:rows + 1])
    np.testing.assert_array_equal(out[0], guard[0])
    np.testing.assert_array_equal(out[rows + 1], guard[rows + 1])
    assert oracle.rel_l2(out[1:rows + 1], oracle.fastconv(x, rep)) <= RTOL
    X = Fftm(rows, n, fft_fwd, 1.0)(x)
    assert oracle.rel_l2(X, oracle.fft_rows(x, -1)) <= RTOL


def test_single_row_at_an_odd_stride(oracle):
    rng = np.random.default_rng(4)
    big = crandn(rng, (3, 4096 + 3))
    x = big[1:2, 1:4097]  # one row, not 16-byte aligned
    y = Fftm(1, 4096, fft_inv, 0.25)(x)
    assert oracle.rel_l2(y, oracle.fft_rows(x, +1, 0.25)) <= RTOL


@pytest.mark.parametrize("scale", [0.0, -1.5])
def test_zero_and_negative_scale(oracle, scale):
    rng = np.random.default_rng(5)
    x = crandn(rng, (8, 2048))
    y = Fftm(8, 2048, fft_fwd, scale)(x)
    if scale == 0.0:
        assert not y.any()
    else:
        assert oracle.rel_l2(y, scale * oracle.fft_rows(x, -1)) <= RTOL


def test_refused_calls():
    rng = np.random.default_rng(6)
    fc = Fastconv(crandn(rng, (4, 512)), 8)  # one replica row per data row, 4 rows
    with pytest.raises(FcbError):
        fc(crandn(rng, (5, 512)))  # more rows than replica rows
    f = Fftm(8, 512, fft_fwd, 1.0)
    with pytest.raises(ValueError):
        f(crandn(rng, (8, 256)))  # row length differs from the plan
    with pytest.raises(FcbError):
        f(crandn(rng, (9, 512)))  # more rows than planned
    with pytest.raises(ValueError):
        Fftm(8, 512, 0, 1.0)  # not a direction tag
