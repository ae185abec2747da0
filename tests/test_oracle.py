"""The CPU oracle is pinned before it is trusted: against the reference's own
golden vectors (tests/fft_ext/data), against outputs of the reference library
itself (fixtures made by tests/golden/make_golden.py), and across its own
independent methods (O(N^2) DFT, FP64 FFT, numpy)."""
import numpy as np
import pytest

from conftest import crandn


@pytest.mark.parametrize("k", range(1, 9))
def test_oracle_dft_matches_reference_golden_vectors(oracle, golden_fft_ext, k):
    # tests/fft_ext/fft_ext.cpp:160 applies Fft(size, scale) and requires < -100 dB
    x = golden_fft_ext[f"f{k}_in"]
    want = golden_fft_ext[f"f{k}_out"]
    scale = float(golden_fft_ext[f"f{k}_scale"])
    got = oracle.dft_rows(x, -1, scale, method=0)[0]
    assert oracle.error_db(want, got) < -100
    # the FFT method agrees too (it falls back to the DFT for non-powers of two)
    got2 = oracle.dft_rows(x, -1, scale, method=1)[0]
    assert oracle.error_db(want, got2) < -100


@pytest.mark.parametrize("n", [1, 2, 3, 8, 18, 19, 64, 68, 252, 256, 768, 1024])
def test_oracle_methods_agree(oracle, n):
    rng = np.random.default_rng(n)
    x = crandn(rng, (3, n)).astype(np.complex128)
    for e in (-1, +1):
        a = oracle.dft_rows(x, e, 1.0, method=0)
        b = oracle.dft_rows(x, e, 1.0, method=1)
        c = oracle.fft_rows(x, e, 1.0)
        assert oracle.rel_l2(a, c) < 1e-12
        assert oracle.rel_l2(b, c) < 1e-12


@pytest.mark.parametrize("n", [64, 128, 256, 512])
def test_oracle_matches_reference_fftm(oracle, golden_ref, n):
    x = golden_ref[f"fftm_in_{n}"]
    fwd = oracle.fft_rows(x, -1, 1.0)
    inv = oracle.fft_rows(x, +1, 1.0 / n)
    assert oracle.error_db(golden_ref[f"fftm_fwd_{n}"], fwd) < -100
    assert oracle.error_db(golden_ref[f"fftm_inv_{n}"], inv) < -100
    assert oracle.rel_l2(golden_ref[f"fftm_fwd_{n}"], fwd) < 1e-6


def test_oracle_matches_reference_fastconv(oracle, golden_ref):
    x, rep = golden_ref["fc_in"], golden_ref["fc_rep"]
    for method in ("numpy", "fft", "dft"):
        y = oracle.fastconv(x, rep, method=method)
        assert oracle.error_db(golden_ref["fc_phased"], y) < -100
        assert oracle.rel_l2(y, golden_ref["fc_phased"]) < 1e-6
    # the reference's phased and fused forms agree with each other
    assert oracle.error_db(golden_ref["fc_phased"], golden_ref["fc_fused"]) < -100


def test_oracle_shift_kernel_identity(oracle, golden_ref):
    # tests/fastconv.cpp:341-366: weights = 2 * delta(shift) -> output = 2 * input shifted
    x, rep, shift = golden_ref["shift_in"], golden_ref["shift_rep"], 2
    y = oracle.fastconv(x, rep)
    n = x.shape[1]
    assert oracle.error_db(2 * x[:, : n - shift], y[:, shift:]) < -100
    assert oracle.error_db(golden_ref["shift_fused"], y) < -100


def test_oracle_matrix_of_coefficients(oracle, golden_ref):
    y = oracle.fastconv(golden_ref["mat_in"], golden_ref["mat_rep"])
    assert oracle.error_db(golden_ref["mat_fused"], y) < -100


def test_error_db_known_answers(oracle):
    a = np.array([1 + 1j, 2, -3j], dtype=np.complex128)
    assert oracle.error_db(a, a) == -201.0
    # negated: max |2a|^2 / (2 max|a|^2) = 4*9/(2*9) = 2 -> 10 log10(2)
    assert abs(oracle.error_db(a, -a) - 10 * np.log10(2.0)) < 1e-12
    b = a.copy()
    b[0] = np.nan
    assert oracle.error_db(a, b) == 201.0


def test_fp32_cpu_baseline_accuracy(oracle, golden_ref):
    x, rep = golden_ref["fc_in"], golden_ref["fc_rep"]
    y = oracle.fastconv_f32(x, rep)
    ref = oracle.fastconv(x, rep)
    assert oracle.rel_l2(y, ref) < 2e-6


@pytest.mark.skipif(not __import__("os").path.exists(
    __import__("os").path.join(__import__("os").path.dirname(__file__), "..", "oracle", "_ref", "ref_driver")),
    reason="reference build (oracle/_ref) not present")
def test_reference_build_matches_oracle(oracle, tmp_path):
    import subprocess
    rng = np.random.default_rng(7)
    rows, n = 3, 128
    x = crandn(rng, (rows, n))
    rep = crandn(rng, (n,))
    x.tofile(tmp_path / "in.bin")
    rep.tofile(tmp_path / "rep.bin")
    subprocess.run([oracle.REF_DRIVER, "phased", str(rows), str(n), "-", str(tmp_path / "in.bin"),
                    str(tmp_path / "rep.bin"), str(tmp_path / "out.bin")], check=True)
    y = np.fromfile(tmp_path / "out.bin", dtype=np.complex64).reshape(rows, n)
    assert oracle.rel_l2(y, oracle.fastconv(x, rep)) < 1e-6
