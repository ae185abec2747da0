"""Generate the golden fixtures under tests/golden/ (run in a container that has
the reference tree; the fixtures themselves are committed and travel).

1. fft_ext_cc.npz -- the reference's own complex->complex golden vectors
   (tests/fft_ext/data/ccfftop_f1..f8, format read as in
   tests/fft_ext/fft_ext.cpp:118-160: header "size scale ntimes", then per line
   "re_in,im_in  re_out,im_out"), converted to arrays.
2. ref_outputs.npz -- outputs of the REFERENCE library itself, built here from
   its sources with its generic FP64 DFT backend (oracle/_ref/ref_driver, built
   by oracle/Makefile), on seeded inputs:
     fwd / inv Fftm on 5 x N rows (tests/fftm.cpp:62-399 shapes),
     phased fast convolution 8 x 2048 with an LFM replica (TBP 100) -- rows of
     the 64 x 2048 CPU configuration,
     the shift-kernel fused fast convolution 16 x 64 (tests/fastconv.cpp:341-366),
     the matrix-of-coefficients form 16 x 64 (tests/fastconv.cpp:213-246).
3. matched_filter_ref.txt -- the printed output of the reference's radar
   matched-filter example (share/examples/radar/matched_filter.cpp, 100
   Doppler rows x 1000 samples), built by oracle/Makefile on the reference's
   generic backend (oracle/_ref/matched_filter).

Usage: python tests/golden/make_golden.py [/path/to/reference]
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# the reference checkout: the argument, else $OPENVSIP_REF, else a directory
# named "reference" beside this repository
REF = (sys.argv[1] if len(sys.argv) > 1 else None) or os.environ.get("OPENVSIP_REF") or \
    os.path.join(os.path.dirname(ROOT), "reference")
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


def parse_cc(path):
    with open(path) as f:
        head = f.readline().split()
        size, scale, ntimes = int(head[0]), float(head[1]), int(head[2])
        xin, xout = [], []
        for _ in range(size):
            line = f.readline()
            a, b = line.split()
            ar, ai = a.split(",")
            br, bi = b.split(",")
            xin.append(complex(float(ar), float(ai)))
            xout.append(complex(float(br), float(bi)))
    return size, scale, ntimes, np.array(xin), np.array(xout)


def fft_ext():
    out = {}
    for k in range(1, 9):
        size, scale, ntimes, xin, xout = parse_cc(os.path.join(REF, "tests", "fft_ext", "data", f"ccfftop_f{k}"))
        out[f"f{k}_scale"] = np.float64(scale)
        out[f"f{k}_in"] = xin
        out[f"f{k}_out"] = xout
    np.savez_compressed(os.path.join(HERE, "fft_ext_cc.npz"), **out)


def run(mode, rows, cols, x, rep=None, scale=None):
    with tempfile.TemporaryDirectory() as d:
        fin, frep, fout = (os.path.join(d, n) for n in ("in.bin", "rep.bin", "out.bin"))
        np.ascontiguousarray(x, dtype=np.complex64).tofile(fin)
        if rep is not None:
            np.ascontiguousarray(rep, dtype=np.complex64).tofile(frep)
        args = [DRIVER, mode, str(rows), str(cols), "-" if scale is None else repr(scale), fin,
                frep if rep is not None else "-", fout]
        subprocess.run(args, check=True)
        return np.fromfile(fout, dtype=np.complex64).reshape(rows, cols)


def lfm(length, tbp, n_out):
    n = np.arange(length)
    c = np.exp(1j * np.pi * tbp * (n / length - 0.5) ** 2)
    out = np.zeros(n_out, dtype=np.complex128)
    out[:length] = c
    return out


def ref_outputs():
    rng = np.random.default_rng(20240601)
    out = {}
    for n in (64, 128, 256, 512):
        x = (rng.uniform(-1, 1, (5, n)) + 1j * rng.uniform(-1, 1, (5, n))).astype(np.complex64)
        out[f"fftm_in_{n}"] = x
        out[f"fftm_fwd_{n}"] = run("fwd", 5, n, x, scale=1.0)
        out[f"fftm_inv_{n}"] = run("inv", 5, n, x, scale=1.0 / n)
    # phased fast convolution on 8 rows of the 64 x 2048 CPU configuration
    n = 2048
    x = ((rng.standard_normal((8, n)) + 1j * rng.standard_normal((8, n)))).astype(np.complex64)
    rep = np.conj(np.fft.fft(lfm(n, 100.0, n))).astype(np.complex64)
    out["fc_in"] = x
    out["fc_rep"] = rep
    out["fc_phased"] = run("phased", 8, n, x, rep)
    out["fc_fused"] = run("fused", 8, n, x, rep)
    # shift kernel: weights delta at `shift` with scale 2 -> spectrum t2f(weights)
    n, shift = 64, 2
    w = np.zeros(n, dtype=np.complex128)
    w[shift] = 2.0
    wspec = np.fft.fft(w).astype(np.complex64)
    ramp = np.tile(np.arange(n, dtype=np.float32), (16, 1)).astype(np.complex64)
    out["shift_in"] = ramp
    out["shift_rep"] = wspec
    out["shift_fused"] = run("fused", 16, n, ramp, wspec)
    # matrix of coefficients: row i weights delta at shift, scale 2*(1+i/n)
    wm = np.zeros((16, n), dtype=np.complex128)
    for i in range(16):
        wm[i, shift] = 2.0 * (1 + i / n)
    wmspec = np.fft.fft(wm, axis=1).astype(np.complex64)
    xm = (rng.standard_normal((16, n)) + 1j * rng.standard_normal((16, n))).astype(np.complex64)
    out["mat_in"] = xm
    out["mat_rep"] = wmspec
    out["mat_fused"] = run("fusedm", 16, n, xm, wmspec)
    np.savez_compressed(os.path.join(HERE, "ref_outputs.npz"), **out)


def matched_filter():
    prog = os.path.join(ROOT, "oracle", "_ref", "matched_filter")
    out = subprocess.run([prog], capture_output=True, text=True, check=True).stdout
    with open(os.path.join(HERE, "matched_filter_ref.txt"), "w") as f:
        f.write(out)


if __name__ == "__main__":
    fft_ext()
    if not os.path.exists(DRIVER) or not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "matched_filter")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REF}"], check=True)
    ref_outputs()
    matched_filter()
    print("fixtures written to", HERE)
