"""Autotuner for the fcb200 kernels.

What it chooses (measured on the device with CUDA events, never guessed):

* For each row length and kind (forward Fftm, inverse Fftm, fused fastconv),
  the tile schedule of the row kernel: CTAs of 128 threads (4096 samples per
  CTA, four CTAs per SM; rows of 256 .. 8192 samples), 256 threads (8192
  samples, two per SM) or 512 threads (16384 samples, one per SM; rows of 4096
  samples and more), or 256 threads with 64 samples each (value -256, rows of
  16384 samples).  Rows longer than one CTA's samples split over a
  thread-block cluster.  The choice is installed with fcb_tune_set and applies
  to plans made afterwards.
* For the batched launch: the kernel (CTAs of 256 or 512 threads with 32
  samples each, clusters of 4 x 256 or 2 x 512 threads for 32768-sample rows;
  or -256, the wide kernel: 256 threads with 64 samples each for rows of
  16384 and 32768, clusters of 2 x 256 for 32768) and the job order (longest
  rows first, or as given).

The reference's analogue is FFTW's planning rigor chosen per Fftm object
(src/ovxx/fftw/fft.cpp:44-52).  Results are cached as JSON keyed by GPU name,
at $FCB200_TUNE_CACHE or ~/.cache/openvsip_b200/tuning.json.
"""
from __future__ import annotations

import json
import os

from . import _lib
from ._lib import lib

KINDS = {"forward": 0, "inverse": 1, "fastconv": 2}
VARIANT_MIN_N = 256  # below this every length has only the 256-thread kernel


def variants(n: int) -> tuple:
    """Kernel variants the library has at row length n: CTA sizes with 32
    samples per thread, and -256 (256 threads x 64 samples) at 16384 and
    32768 (a cluster of two such CTAs)."""
    out = [256]
    if 256 <= n <= 8192:
        out.insert(0, 128)
    if n >= 4096:
        out.append(512)
    if n in (16384, 32768):
        out.append(-256)
    return tuple(out)


def cache_path() -> str:
    return os.environ.get("FCB200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "openvsip_b200", "tuning.json"))


def _gpu_key() -> str:
    import torch
    return torch.cuda.get_device_name(0)


def _time_ms(fn, reps: int) -> float:
    import torch
    for _ in range(3):
        fn()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def time_plan(kind: str, n: int, threads: int, samples: int = 1 << 24, reps: int = 10) -> float:
    """Milliseconds per call of one plan of `kind` over `samples` samples."""
    import numpy as np
    import torch

    from .vsip import Fastconv, Fftm, fft_fwd, fft_inv
    rows = max(1, samples // n)
    _lib.check(lib().fcb_tune_set(n, KINDS[kind], threads))
    x = torch.randn(rows, n, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    if kind == "fastconv":
        plan = Fastconv(np.ones(n, dtype=np.complex64), rows)
    else:
        plan = Fftm(rows, n, fft_fwd if kind == "forward" else fft_inv, 1.0)
    return _time_ms(lambda: plan(x, y), reps)


def tune_plans(lengths=(1024, 4096, 8192, 16384, 32768, 65536), kinds=tuple(KINDS), samples: int = 1 << 24) -> dict:
    """Pick the CTA size per (kind, length); installs and returns the choices."""
    out = {}
    for kind in kinds:
        for n in lengths:
            if n < VARIANT_MIN_N:
                continue
            times = {t: time_plan(kind, n, t, samples) for t in variants(n)}
            best = min(times, key=times.get)
            _lib.check(lib().fcb_tune_set(n, KINDS[kind], best))
            out[f"{kind}:{n}"] = {"threads": best, "ms": times}
    return out


def tune_batch(make_batch, orders=("longest_first", "as_given"), threads=(256, 512, -256), reps: int = 5) -> dict:
    """make_batch(threads, order) -> Batch with its jobs set; returns the best
    {"threads", "order", "ms"} and all timings."""
    results = {}
    for t in threads:
        for o in orders:
            b = make_batch(t, o)
            results[(t, o)] = _time_ms(lambda: (b.run(), b.sync()), reps)
            del b
    (t, o), ms = min(results.items(), key=lambda kv: kv[1])
    return {"threads": t, "order": o, "ms": ms,
            "all": {f"{k[0]}/{k[1]}": v for k, v in results.items()}}


def save(results: dict, path: str | None = None) -> str:
    path = path or cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data.setdefault(_gpu_key(), {}).update(results)
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    return path


def load(path: str | None = None) -> dict:
    """Install cached plan choices for this GPU; returns the cached entries."""
    path = path or cache_path()
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        data = json.load(f).get(_gpu_key(), {})
    for key, v in data.items():
        if ":" in key and isinstance(v, dict) and "threads" in v:
            kind, n = key.split(":")
            if kind in KINDS:
                lib().fcb_tune_set(int(n), KINDS[kind], int(v["threads"]))
    return data
