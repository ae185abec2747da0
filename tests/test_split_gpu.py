"""The split variant of the fused fast convolution at 32768 samples (fcb_tune_set
value -2): one 256-thread CTA per row runs the row as the two 16384-sample
halves of a radix-2 decimation in frequency, one after the other, with the
waiting half held in tensor memory.  Checked against the FP64 oracle (relative
L2 <= 2e-6) for a shared replica and for a matrix of coefficients, in place,
on strided rows and fewer rows than planned, with the rows around the call
left untouched, and against the cluster variant's result."""
import numpy as np
import pytest

from conftest import crandn, pinned_variant
from openvsip_b200 import Fastconv, synth

pytestmark = pytest.mark.gpu
RTOL = 2e-6
N = 32768


@pytest.mark.parametrize("rows", [1, 3, 20])
def test_split_fastconv_vs_fp64(oracle, rows):
    rng = np.random.default_rng(900 + rows)
    x = crandn(rng, (rows, N))
    rep = crandn(rng, (N,))
    w = crandn(rng, (rows, N))
    with pinned_variant(N, 2, -2):
        fc = Fastconv(rep, rows)
        info = fc.info()
        assert info["threads"] == 256 and info["cluster_ctas"] == 1
        guard = crandn(rng, (rows + 2, N))
        out = guard.copy()
        fc(x, out[1:rows + 1])
        np.testing.assert_array_equal(out[0], guard[0])
        np.testing.assert_array_equal(out[rows + 1], guard[rows + 1])
        assert oracle.rel_l2(out[1:rows + 1], oracle.fastconv(x, rep)) <= RTOL
        # matrix of coefficients: one replica spectrum per row
        assert oracle.rel_l2(Fastconv(w, rows)(x), oracle.fastconv(x, w)) <= RTOL


def test_split_fastconv_device_in_place_strided_fewer_rows(oracle):
    import torch
    rows, pad = 12, 40
    rng = np.random.default_rng(33)
    big = crandn(rng, (rows, N + pad))
    chirp = synth.lfm_chirp(N, 700.0, N).astype(np.complex64)
    spec = np.conj(np.fft.fft(chirp.astype(np.complex128))).astype(np.complex64)
    with pinned_variant(N, 2, -2):
        fc = Fastconv(chirp, rows + 5, kind="matched")  # replica built in FP64 on the GPU
        d = torch.from_numpy(big).cuda()
        view = d[:, :N]
        fc.in_place(view)
        torch.cuda.synchronize()
        got = d.cpu().numpy()
    assert oracle.rel_l2(got[:, :N], oracle.fastconv(big[:, :N], spec)) <= RTOL
    np.testing.assert_array_equal(got[:, N:], big[:, N:])  # the padding is untouched


def test_split_matches_cluster_variant(oracle):
    rows = 8
    rng = np.random.default_rng(5)
    x = crandn(rng, (rows, N))
    rep = crandn(rng, (N,))
    with pinned_variant(N, 2, -2):
        a = Fastconv(rep, rows)(x)
    with pinned_variant(N, 2, 512):
        b = Fastconv(rep, rows)(x)
    want = oracle.fastconv(x, rep)
    assert oracle.rel_l2(a, want) <= RTOL and oracle.rel_l2(b, want) <= RTOL
    assert oracle.rel_l2(a, b) <= 2 * RTOL
