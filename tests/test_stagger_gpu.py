"""Kernels with one CTA per SM (512 threads of 32 samples, and 256 threads of 64
samples) run the two halves of each CTA out of phase through the sub-problem
stages.  These cases pin those variants at lengths where a CTA holds several
rows or a cluster shares one, with row counts that leave the last CTA partly
empty (its idle rows still take part in every barrier), in all three modes,
against FP64 (relative L2 <= 2e-6)."""
import numpy as np
import pytest

from conftest import crandn, pinned_variant
from openvsip_b200 import Fastconv, Fftm, fft_fwd, fft_inv

pytestmark = pytest.mark.gpu
RTOL = 2e-6


@pytest.mark.parametrize("n,rows,threads", [(4096, 5, 512), (4096, 7, 512), (8192, 3, 512), (16384, 3, 512),
                                            (16384, 1, -256), (16384, 3, -256), (32768, 3, 512), (32768, 1, -256),
                                            (32768, 3, -256)])
def test_staggered_variants_with_idle_rows(oracle, n, rows, threads):
    rng = np.random.default_rng(n + rows + threads)
    x = crandn(rng, (rows, n))
    rep = crandn(rng, (n,))
    with pinned_variant(n, 0, threads), pinned_variant(n, 1, threads), pinned_variant(n, 2, threads):
        f = Fftm(rows, n, fft_fwd, 1.0)
        assert f.info()["threads"] == abs(threads)
        assert oracle.rel_l2(f(x), oracle.fft_rows(x, -1)) <= RTOL
        y = Fftm(rows, n, fft_inv, 1.0 / n)(x)
        assert oracle.rel_l2(y, oracle.fft_rows(x, +1, 1.0 / n)) <= RTOL
        guard = crandn(rng, (rows + 1, n))
        out = guard.copy()
        Fastconv(rep, rows)(x, out[:rows])
        np.testing.assert_array_equal(out[rows], guard[rows])  # the row after the call is untouched
        assert oracle.rel_l2(out[:rows], oracle.fastconv(x, rep)) <= RTOL
