"""The SSAR benchmark's kernel-1 transforms at the application's own sizes.

The application itself (share/apps/ssar) reads its inputs from HDF5 files and
HDF5 is not available, so it is not built.  Its Fftm objects, though, are the
kind this library replaces, and they are declared with shapes, axes, directions
and scales of their own (share/apps/ssar/kernel1.hpp:304-312 and 427-433, used
at :691-731 and :788-790; the scale-3 sizes n = 1072, mc = 480, m = 1144,
nx = 756 of share/apps/ssar/data/dims.txt).  This test runs the same sequence
of transforms on seeded synthetic data: column and row Fftm, forward and
inverse, by value and in place, with the kernel's scales, all of non-power-of-
two length (so through Bluestein's algorithm).  Each step is checked against
FP64 on that step's own input (relative L2 <= 2e-6)."""
import numpy as np
import pytest

from conftest import crandn
from openvsip_b200 import Fftm, col, fft_fwd, fft_inv, row

pytestmark = pytest.mark.gpu
RTOL = 2e-6
N, MC, M, NX = 1072, 480, 1144, 756


def _col_ref(oracle, x, exponent, scale):
    return oracle.fft_rows(np.asarray(x).T, exponent, scale).T


def test_ssar_kernel1_transform_sequence(oracle):
    rng = np.random.default_rng(1072)
    # ft_fftm_: Fftm<C, C, col, fft_fwd, by_value>(Domain<2>(n, mc), 1), :427, :691
    s = crandn(rng, (N, MC))
    ft = Fftm(N, MC, fft_fwd, 1.0, axis=col)
    S = ft(s)
    assert oracle.rel_l2(S, _col_ref(oracle, s, -1, 1.0)) <= RTOL
    filt = crandn(rng, (N, MC))
    s_filt = (filt * S).astype(np.complex64)

    # compr_fftm_: Fftm<C, C, row, fft_fwd, by_reference>(Domain<2>(n, mc), m / mc), :429, :697
    compr = Fftm(N, MC, fft_fwd, M / MC, axis=row)
    fs = s_filt.copy()
    compr.in_place(fs)
    assert oracle.rel_l2(fs, oracle.fft_rows(s_filt, -1, M / MC)) <= RTOL

    # decompr_fftm_: Fftm<C, C, row, fft_inv, by_value>(Domain<2>(n, m), 1/m), :430, :720
    fs_padded = np.zeros((N, M), dtype=np.complex64)
    fs_padded[:, (M - MC) // 2:(M - MC) // 2 + MC] = fs
    decompr = Fftm(N, M, fft_inv, 1.0 / M, axis=row)
    d = decompr(fs_padded)
    assert oracle.rel_l2(d, oracle.fft_rows(fs_padded, +1, 1.0 / M)) <= RTOL

    # st_fftm_: Fftm<C, C, row, fft_fwd, by_value>(Domain<2>(n, m), 1), :428, :731
    st = Fftm(N, M, fft_fwd, 1.0, axis=row)
    fsm = st(d)
    assert oracle.rel_l2(fsm, oracle.fft_rows(d, -1, 1.0)) <= RTOL

    # ifftmc_: Fftm<C, C, col, fft_inv, by_reference>(Domain<2>(nx, m), 1/nx), :433, :788
    F = crandn(rng, (NX, M))
    ifc = Fftm(NX, M, fft_inv, 1.0 / NX, axis=col)
    Fc = F.copy()
    ifc.in_place(Fc)
    assert oracle.rel_l2(Fc, _col_ref(oracle, F, +1, 1.0 / NX)) <= RTOL

    # ifftmr_: Fftm<C, C, row, fft_inv, by_reference>(Domain<2>(nx, m), 1/m), :432, :790
    ifr = Fftm(NX, M, fft_inv, 1.0 / M, axis=row)
    spatial = Fc.copy()
    ifr.in_place(spatial)
    assert oracle.rel_l2(spatial, oracle.fft_rows(Fc, +1, 1.0 / M)) <= RTOL


def test_ssar_kernel1_transforms_on_the_device(oracle):
    # the same objects on device-resident data, in one stream, as a GPU pipeline would hold them
    import torch
    rng = np.random.default_rng(480)
    s = crandn(rng, (N, M))
    st = Fftm(N, M, fft_fwd, 1.0, axis=row)
    decompr = Fftm(N, M, fft_inv, 1.0 / M, axis=row)
    d = torch.from_numpy(s).cuda()
    y = decompr(st(d))  # forward then inverse with 1/m: the identity up to rounding
    torch.cuda.synchronize()
    assert oracle.rel_l2(y.cpu().numpy(), s) <= RTOL
