"""The drop-in boundary exercised through the reference's own public API.

openvsip_b200/plugin/_bin holds programs built (where the reference sources
exist) from the reference's unmodified tests/fastconv.cpp and tests/fftm.cpp
with the B200 plugin injected (-include ovxx_fcb200.hpp), and plugin_check.cpp,
which runs the phased, fused and matrix-of-coefficients forms through vsip::Fftm
/ vmmul on seeded data.  The reference tests self-check (test_assert aborts,
-100 dB thresholds); FCB200_TRACE shows that the B200 backend, not the
reference's generic one, ran."""
import os
import subprocess

import numpy as np
import pytest

from conftest import HAS_GPU, crandn

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "openvsip_b200", "plugin", "_bin")


def _prog(name):
    p = os.path.join(BIN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not built (needs the reference sources at build time)")
    return p


def _run(args, **kw):
    env = dict(os.environ, FCB200_TRACE="1")
    return subprocess.run(args, capture_output=True, text=True, env=env, timeout=600, **kw)


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_plugin_fails_loudly_without_gpu():
    r = _run([_prog("fastconv_test")])
    assert r.returncode != 0
    assert "fcb200" in r.stderr and "device" in r.stderr


@pytest.mark.gpu
def test_reference_fastconv_test_on_b200():
    r = _run([_prog("fastconv_test")])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "[fcb200] Fftm<fwd>" in r.stderr
    assert "[fcb200] fused fastconv" in r.stderr and "vector weights" in r.stderr
    assert "matrix weights" in r.stderr
    assert "[fcb200] Fft<1,fwd>" in r.stderr  # the replica's t2f (1-D vsip::Fft)


@pytest.mark.gpu
def test_reference_fftm_test_on_b200():
    # rows and columns, powers of two and not (18, 68, 252: Bluestein), and
    # test_real's real <-> complex Fftm along columns (16, 128, 242)
    r = _run([_prog("fftm_test")])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "[fcb200] Fftm<fwd>" in r.stderr and "[fcb200] Fftm<inv>" in r.stderr
    assert "[fcb200] Fftm<fwd, col> 68 x" in r.stderr and "[fcb200] Fftm<inv, col>" in r.stderr
    assert "Fftm<fwd> 5 x 252" in r.stderr or "x 252 scale" in r.stderr
    for n in (16, 128, 242):
        assert f"[fcb200] Fftm<real->complex, col> n {n} x 5" in r.stderr
        assert f"[fcb200] Fftm<complex->real, col> n {n} x 5" in r.stderr


@pytest.mark.gpu
def test_reference_fft_test_on_b200():
    # tests/fft.cpp: 1-D complex FFTs by reference and by value, interleaved and
    # split storage, at 64, 128, 256, 512 and at 68, 252, 17 (Bluestein), each
    # checked by the test itself; its real cases stay on the generic backend
    r = _run([_prog("fft_test")])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    for n in (64, 256, 512, 68, 252, 17):
        assert f"[fcb200] Fft<1,fwd> {n} " in r.stderr, n
        assert f"[fcb200] Fft<1,inv> {n} " in r.stderr, n


@pytest.mark.gpu
def test_reference_matched_filter_example_on_b200():
    # share/examples/radar/matched_filter.cpp: a matched-filter bank over 100
    # Doppler shifts x 1000 delays (coefficients by a forward Fftm, output by
    # an inverse Fftm of vmmul<0>); its printed delays must equal those of the
    # same program on the reference's own backend (tests/golden/matched_filter_ref.txt)
    r = _run([_prog("ex_matched_filter")])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    want = open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "matched_filter_ref.txt")).read()
    assert r.stdout == want
    assert "[fcb200] Fftm<fwd> 100 x 1000" in r.stderr and "[fcb200] Fftm<inv> 100 x 1000" in r.stderr


@pytest.mark.gpu
def test_reference_fft2d_test_on_b200():
    # tests/fft2d.cpp: forward and inverse 2-D complex FFTs by reference, by
    # value and in place, scales 1, 1/4 and 1/N, at 8 x 8 and at the sizes that
    # are not powers of two (2 x 2, 1 x 1, 2 x 1, 4 x 8, 8 x 128, 5 x 7, 24 x 48,
    # 1 x 5), each checked by the test itself at -100 dB
    r = _run([_prog("fft2d_test")])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    for shape in ("8 x 8", "5 x 7", "24 x 48", "8 x 128", "1 x 5"):
        assert f"[fcb200] Fft<2,fwd> {shape}" in r.stderr, shape
        assert f"[fcb200] Fft<2,inv> {shape}" in r.stderr, shape


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fftm_unaligned", "fft_ip_subview", "fft_temp_view"])
def test_reference_fftm_regressions_on_b200(name):
    # tests/regressions: unaligned and gapped rows in interleaved and split
    # storage, in-place subviews, temporary views (rows and columns)
    r = _run([_prog("reg_" + name)])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "[fcb200] Fftm<" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fft_inter_split", "fft_unaligned", "fft_expr_arg"])
def test_reference_fft_regressions_on_b200(name):
    # tests/regressions for the 1-D vsip::Fft: interleaved <-> split storage by
    # reference, by value and of expressions (256), unaligned subviews in and
    # out of place (256), an expression argument with a decimated subview
    r = _run([_prog("reg_" + name)])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "[fcb200] Fft<1," in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("rows,cols", [(64, 4096), (8, 32768), (256, 4096)])
def test_plugin_forms_match_oracle(oracle, tmp_path, rows, cols):
    rng = np.random.default_rng(rows + cols)
    x = crandn(rng, (rows, cols))
    w = crandn(rng, (cols,))
    x.tofile(tmp_path / "in.bin")
    w.tofile(tmp_path / "w.bin")
    r = _run([_prog("plugin_check"), str(rows), str(cols), str(tmp_path / "in.bin"), str(tmp_path / "w.bin"),
              str(tmp_path / "out")])
    assert r.returncode == 0, r.stderr[-2000:]
    want = oracle.fastconv(x, w)
    for form in ("phased", "fused"):
        y = np.fromfile(tmp_path / f"out.{form}.bin", dtype=np.complex64).reshape(rows, cols)
        assert oracle.rel_l2(y, want) <= 2e-6, form
    wm = (w[None, :] * (1 + np.arange(rows, dtype=np.float32)[:, None] / rows)).astype(np.complex64)
    ym = np.fromfile(tmp_path / "out.fusedm.bin", dtype=np.complex64).reshape(rows, cols)
    assert oracle.rel_l2(ym, oracle.fastconv(x, wm)) <= 2e-6
    # the cached plan for unchanged weights (256 x 4096: an 8 MB weight matrix,
    # compared on several threads), a new one after one weight changed
    np.testing.assert_array_equal(np.fromfile(tmp_path / "out.fusedm2.bin", dtype=np.complex64).reshape(rows, cols), ym)
    wm[-1, -1] *= 2
    ym3 = np.fromfile(tmp_path / "out.fusedm3.bin", dtype=np.complex64).reshape(rows, cols)
    assert oracle.rel_l2(ym3[-1:], oracle.fastconv(x[-1:], wm[-1:])) <= 2e-6
    np.testing.assert_array_equal(ym3[:-1], ym[:-1])
    assert r.stderr.count("fused fastconv") >= 4
    # the 2-D vsip::Fft forward (by reference) and inverse (by value, scale 1 / (rows cols))
    y2 = np.fromfile(tmp_path / "out.fft2d.bin", dtype=np.complex64).reshape(rows, cols)
    assert oracle.rel_l2(y2, np.fft.fft2(x.astype(np.complex128))) <= 2e-6
    rt = np.fromfile(tmp_path / "out.fft2d_rt.bin", dtype=np.complex64).reshape(rows, cols)
    assert oracle.rel_l2(rt, x) <= 2e-6
    assert f"[fcb200] Fft<2,fwd> {rows} x {cols}" in r.stderr and f"[fcb200] Fft<2,inv> {rows} x {cols}" in r.stderr
