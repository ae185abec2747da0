"""2-D FFT (two transposing row passes) against the FP64 oracle, including the
4096 x 4096 forward + inverse case, at relative L2 <= 2e-6."""
import numpy as np
import pytest

from conftest import crandn
from openvsip_b200 import Fft2d, fft_fwd, fft_inv, synth

pytestmark = pytest.mark.gpu
RTOL = 2e-6


@pytest.mark.parametrize("rows,cols", [(64, 64), (128, 1024), (2048, 256), (16384, 64), (64, 16384)])
def test_fft2d_vs_fp64(oracle, rows, cols):
    rng = np.random.default_rng(rows * 7 + cols)
    x = crandn(rng, (rows, cols))
    y = Fft2d(rows, cols, fft_fwd)(x)
    want = np.fft.fft2(x.astype(np.complex128))
    assert oracle.rel_l2(y, want) <= RTOL
    z = Fft2d(rows, cols, fft_inv, 1.0 / (rows * cols))(x)
    assert oracle.rel_l2(z, np.fft.ifft2(x.astype(np.complex128))) <= RTOL


def test_fft2d_4096_forward_inverse_device(oracle):
    import torch
    x = synth.sweep_matrix(4, 4096, 4096)
    dx = torch.from_numpy(x).cuda()
    f = Fft2d(4096, 4096, fft_fwd)
    g = Fft2d(4096, 4096, fft_inv, 1.0 / (4096 * 4096))
    X = f(dx)
    xr = g(X)
    torch.cuda.synchronize()
    want = np.fft.fft2(x.astype(np.complex128))
    assert oracle.rel_l2(X.cpu().numpy(), want) <= RTOL
    assert oracle.rel_l2(xr.cpu().numpy(), x) <= RTOL  # round trip
    # strided rows through the host path
    big = np.zeros((4096, 4096 + 8), dtype=np.complex64)
    big[:, :4096] = x
    Xh = f(big[:, :4096])
    np.testing.assert_array_equal(Xh, X.cpu().numpy())


@pytest.mark.parametrize("rows,cols", [(1, 1), (1, 5), (5, 7), (8, 8), (24, 48), (8, 128), (100, 64), (3, 1000),
                                       (32, 32768), (1024, 12)])
def test_fft2d_other_sizes_vs_fp64(oracle, rows, cols):
    # sizes outside the two-pass transposing path: row pass, transpose, column
    # pass, transpose back; host and device data, in place and out of place
    import torch
    rng = np.random.default_rng(rows * 13 + cols)
    x = crandn(rng, (rows, cols))
    want = np.fft.fft2(x.astype(np.complex128))
    f = Fft2d(rows, cols, fft_fwd, 0.5)
    assert oracle.rel_l2(f(x), 0.5 * want) <= RTOL
    dx = torch.from_numpy(x).cuda()
    f(dx, dx)  # in place on the device
    torch.cuda.synchronize()
    assert oracle.rel_l2(dx.cpu().numpy(), 0.5 * want) <= RTOL
    g = Fft2d(rows, cols, fft_inv, 2.0 / (rows * cols))
    assert oracle.rel_l2(g(dx).cpu().numpy(), x) <= RTOL


def test_fft2d_rejects_unsupported_sizes():
    from openvsip_b200 import FcbError
    for rows, cols in ((0, 8), (8, 40000), (70000, 4)):
        with pytest.raises(FcbError):
            Fft2d(rows, cols, fft_fwd)
