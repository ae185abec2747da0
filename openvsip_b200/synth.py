"""Seeded synthetic pulse-compression workloads (numpy PCG64 generators).

No public dataset is involved: every workload is generated from its seed.

* LFM chirp c[n] = exp(j pi TBP (n/L - 1/2)^2), n < L, zero-padded to N.
* Matched-filter replica spectrum R = conj(FFT_N(c)), computed in FP64 and
  rounded once to complex64.
* cpu_case:      64 x 2048, i.i.d. complex Gaussian (sigma 1 per component),
                 TBP 100.
* large_fastconv: 1024 pulses x 16384 samples, noise plus 8 echoes per pulse
                 a * c[(n - d) mod N], a ~ U[0.1, 1], d ~ U{0..N-1}; TBP 500.
* uneven_jobs:   jobs with pulses ~ U{16..512} and N from
                 {1024, ..., 32768}, each with its own replica (TBP ~ U[50, 1000]).
* sweep_matrix:  rows x N with re, im ~ U[-1, 1].
"""
from __future__ import annotations

import numpy as np

SIZES = (1024, 2048, 4096, 8192, 16384, 32768)


def lfm_chirp(length: int, tbp: float, n_out: int | None = None) -> np.ndarray:
    n_out = length if n_out is None else n_out
    n = np.arange(length, dtype=np.float64)
    out = np.zeros(n_out, dtype=np.complex128)
    out[:length] = np.exp(1j * np.pi * tbp * (n / length - 0.5) ** 2)
    return out


def matched_spectrum(chirp: np.ndarray) -> np.ndarray:
    return np.conj(np.fft.fft(np.asarray(chirp, dtype=np.complex128))).astype(np.complex64)


def cgauss(rng, shape, sigma=1.0) -> np.ndarray:
    out = np.empty(shape, dtype=np.complex64)
    out.real = rng.standard_normal(shape, dtype=np.float32) * sigma
    out.imag = rng.standard_normal(shape, dtype=np.float32) * sigma
    return out


def cpu_case(seed: int = 0, rows: int = 64, n: int = 2048, tbp: float = 100.0) -> dict:
    rng = np.random.default_rng(seed)
    chirp = lfm_chirp(n, tbp, n)
    return {"data": cgauss(rng, (rows, n)), "chirp": chirp, "replica_spectrum": matched_spectrum(chirp)}


def large_fastconv(seed: int = 0, pulses: int = 1024, n: int = 16384, tbp: float = 500.0,
                   echoes: int = 8) -> dict:
    rng = np.random.default_rng(seed)
    chirp = lfm_chirp(n, tbp, n)
    c32 = chirp.astype(np.complex64)
    data = cgauss(rng, (pulses, n))
    delays = rng.integers(0, n, size=(pulses, echoes))
    amps = rng.uniform(0.1, 1.0, size=(pulses, echoes)).astype(np.float32)
    for p in range(pulses):
        row = data[p]
        for e in range(echoes):
            row += amps[p, e] * np.roll(c32, int(delays[p, e]))
    return {"data": data, "chirp": chirp, "replica_spectrum": matched_spectrum(chirp),
            "delays": delays, "amplitudes": amps}


def uneven_jobs(seed: int = 0, njobs: int = 512, pulses=(16, 512), sizes=SIZES,
                tbp=(50.0, 1000.0)) -> list[dict]:
    """Job descriptors (shapes and replica parameters); data is generated per job
    by job_data() so that large mixes need not be materialised on the host."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(njobs):
        jobs.append({"id": j, "pulses": int(rng.integers(pulses[0], pulses[1] + 1)),
                     "n": int(sizes[int(rng.integers(0, len(sizes)))]),
                     "tbp": float(rng.uniform(tbp[0], tbp[1])), "seed": int(rng.integers(0, 2**31))})
    return jobs


def job_data(job: dict) -> np.ndarray:
    return cgauss(np.random.default_rng(job["seed"]), (job["pulses"], job["n"]))


def job_replica(job: dict) -> np.ndarray:
    return lfm_chirp(job["n"], job["tbp"], job["n"])


def sweep_matrix(seed: int, rows: int, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = np.empty((rows, n), dtype=np.complex64)
    out.real = rng.uniform(-1, 1, (rows, n)).astype(np.float32)
    out.imag = rng.uniform(-1, 1, (rows, n)).astype(np.float32)
    return out
