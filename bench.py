"""Benchmark of the fused fast convolution (pulse compression) on B200.

Workload (one GPU): a single large fast convolution, 1024 pulses x 16384
samples complex<float>, complex Gaussian noise plus 8 LFM echoes per pulse,
matched replica of TBP 500.  One step = one fused forward-FFT x replica x
inverse-FFT pass over that batch, inputs resident in HBM (256 MB read+write per
step, larger than the 126 MB L2; two input buffers alternate).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 is launched by torchrun (one rank per GPU); every rank runs its own
batch (weak scaling, no data-path collective), timing is the max over ranks.
Prints one JSON line on rank 0.  Besides the headline it carries blocks for
the phased Impl1op form on the same data ("phased"), the uneven batch of 512
jobs in one persistent launch per step with its jobs partitioned across ranks
("batch"), and, on one GPU, the served Poisson stream ("serve"); --no-batch /
--no-serve leave those out.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PULSES, NSAMP, TBP, ECHOES = 1024, 16384, 500.0, 8
WORKLOAD = f"single large fastconv, {PULSES} pulses x {NSAMP} samples complex<float>, {ECHOES} echoes/pulse, LFM TBP {TBP:g}"


METRIC = "fastconv complex samples/sec & HBM roofline %; p50/p99 latency, at \u22642e-6 rel-L2 vs FP64"


def baseline_metric():
    return METRIC


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def ncu_traffic():
    """Per-launch DRAM bytes of the fused kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "fastconv_1024x16384_ncu.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown", 0x1: "gpu_idle"}

    def __init__(self, device_index: int):
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:
                break
            time.sleep(0.002)

    def __enter__(self):
        if self.nv:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.nv:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def host_info():
    """The GPU box's host: CPU model and thread count (lscpu / os), and whether
    the reference's production FFT library (FFTW3, single precision) is
    installed -- the library and its header are probed, neither is assumed."""
    import ctypes.util
    import glob
    model = None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            if line.startswith("Model name:"):
                model = line.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    headers = []
    for d in ("/usr/include", "/usr/local/include", "/opt/*/include", sys.prefix + "/include"):
        headers += glob.glob(os.path.join(d, "fftw3.h"))
    lib = ctypes.util.find_library("fftw3f")
    return {"cpu_model": model, "nproc": os.cpu_count(), "fftw3f_library": lib, "fftw3_header": headers[0] if
            headers else None, "fftw3_usable": bool(lib and headers)}


def cpu_reference_sample(rows_per_proc: int = 1):
    """The reference library's own CPU path (oracle/_ref, generic DFT backend --
    FFTW3 is not installed) on a bounded sample: nproc processes, each running
    the phased fast convolution on rows_per_proc rows of NSAMP samples."""
    driver = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    cores = os.cpu_count() or 1
    if not os.path.exists(driver):
        return None
    t0 = time.perf_counter()
    procs = [subprocess.Popen([driver, "bench", str(rows_per_proc), str(NSAMP), "1"], stdout=subprocess.PIPE,
                              text=True) for _ in range(cores)]
    outs = [json.loads(p.communicate()[0]) for p in procs]
    wall = time.perf_counter() - t0
    samples = sum(o["samples"] for o in outs)
    return {"value": samples / wall, "unit": "complex samples/s", "cores": cores, "kind": "reference",
            "sample": f"{cores} processes x {rows_per_proc} row x {NSAMP} samples of the workload, phased "
                      f"Fftm->vmmul->Fftm through the reference's own vsip API, generic FP64 DFT backend "
                      f"(FFTW3 not installed; O(N^2)), harness-level process parallelism",
            "seconds": wall}


def plugin_sample(rows: int, cols: int, loops: int):
    """The same workload through the reference's own vsip API with the B200
    plugin included (openvsip_b200/plugin/_bin/plugin_bench, built where the
    reference sources exist): vsip::Matrix blocks in pageable host memory, the
    fused by-value expression and the phased Impl1op form, wall-clock timed."""
    prog = os.path.join(ROOT, "openvsip_b200", "plugin", "_bin", "plugin_bench")
    if not os.path.exists(prog):
        return None
    r = subprocess.run([prog, str(rows), str(cols), str(loops)], capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        return {"error": r.stderr[-300:]}
    o = json.loads(r.stdout.strip().splitlines()[-1])
    return {"value": o["fused_samples_per_s"], "unit": "complex samples/s",
            "phased": {"value": o["phased_samples_per_s"], "unit": "complex samples/s"}, "loops": loops,
            "how": "reference vsip API + B200 plugin (plugin_bench): out = inv_fftm(vmmul<0>(replica, "
                   "for_fftm(data))) by value, one fused B200 pass per call; phased: Fftm by reference, "
                   "vmmul<0> on the host, Fftm; vsip::Matrix blocks in pageable host memory"}


def cpu_port_sample():
    """Fallback when oracle/_ref is absent: the oracle's FP32 radix-2 port."""
    from oracle import oracle
    cores = os.cpu_count() or 1
    rows = 16 * cores
    rng = np.random.default_rng(0)
    x = (rng.standard_normal((rows, NSAMP)) + 1j * rng.standard_normal((rows, NSAMP))).astype(np.complex64)
    rep = np.ones(NSAMP, dtype=np.complex64)
    chunks = np.array_split(np.arange(rows), cores)
    t0 = time.perf_counter()
    ths = [threading.Thread(target=oracle.fastconv_f32, args=(x[c[0]:c[-1] + 1], rep)) for c in chunks]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    wall = time.perf_counter() - t0
    return {"value": rows * NSAMP / wall, "unit": "complex samples/s", "cores": cores, "kind": "port",
            "sample": f"{rows} rows x {NSAMP} samples, oracle FP32 radix-2 port, {cores} threads"}


def rel_l2(y, ref):
    y = np.asarray(y, dtype=np.complex128)
    ref = np.asarray(ref, dtype=np.complex128)
    return float(np.linalg.norm(y - ref) / np.linalg.norm(ref))


def fftw_standin(x, spec, ref):
    """scipy.fft complex64 (pocketfft) fft -> multiply -> ifft with all
    workers: a labelled stand-in for the reference's FFTW3 FP32 path, which is
    not installed.  x: rows of the workload (complex64), spec: the complex64
    replica spectrum, ref: the FP64 result of those rows.  Returns its
    throughput and its own error against FP64 on the same rows as the GPU's."""
    import scipy.fft
    cores = os.cpu_count() or 1
    reps = max(1, 256 // x.shape[0])
    xx = np.concatenate([x] * reps, axis=0)
    scipy.fft.ifft(scipy.fft.fft(xx[:8], axis=1, workers=cores) * spec, axis=1, workers=cores)
    t0 = time.perf_counter()
    for _ in range(3):
        scipy.fft.ifft(scipy.fft.fft(xx, axis=1, workers=cores) * spec, axis=1, workers=cores)
    wall = (time.perf_counter() - t0) / 3
    y = scipy.fft.ifft(scipy.fft.fft(x, axis=1, workers=cores) * spec, axis=1, workers=cores)
    return {"value": xx.shape[0] * x.shape[1] / wall, "unit": "complex samples/s", "cores": cores,
            "rel_l2_vs_fp64": rel_l2(y.astype(np.complex64), ref), "rows_checked": int(x.shape[0]),
            "what": "scipy.fft complex64 fft -> multiply -> ifft, FFTW3 FP32 stand-in (not the reference)"}


# Wall-clock cap of the reference arm.  Its smallest step is one 16384-sample row per host
# process through the reference's O(N^2) DFT backend (several seconds), so K steps of it would
# take far longer than the GPU arm; the arm stops taking steps once this much time has passed.
REF_BUDGET_S = 150.0


def run_reference(args, world, rank):
    if rank != 0:
        return
    steps = []
    cores = os.cpu_count() or 1
    kind = "reference"
    t_begin = time.perf_counter()

    def sample():
        nonlocal kind
        r = cpu_reference_sample(1)
        if r is None:
            r = cpu_port_sample()
            kind = "port"
        return r

    # the reference's CPU code keeps no state between runs: one untimed sample stands for the
    # requested warm-up steps
    warm = 1 if args.warmup > 0 else 0
    for _ in range(warm):
        sample()
    while len(steps) < args.steps and (not steps or time.perf_counter() - t_begin < REF_BUDGET_S):
        steps.append(sample())
    value = statistics.median(s["value"] for s in steps)
    ms = statistics.median(s.get("seconds", 0.0) for s in steps) * 1e3
    line = {"impl": "reference", "metric": baseline_metric(), "value": value, "unit": "complex samples/s",
            "n_gpus": args.gpus, "steps": len(steps), "warmup": warm, "ms_per_step": ms,
            "steps_requested": args.steps, "warmup_requested": args.warmup,
            "note": f"steps stop after {REF_BUDGET_S:.0f} s of wall time; value is the median step",
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": WORKLOAD + " (bounded sample per step)", "parallelism": f"{cores} host processes"},
            "cpu_baseline": {"value": value, "unit": "complex samples/s", "cores": cores, "kind": kind,
                             "sample": steps[-1]["sample"], "host": host_info()},
            "e2e": {"value": value, "unit": "complex samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _time_calls(fn, steps, stream):
    """Mean milliseconds per call of fn over `steps` back-to-back calls (CUDA
    events on `stream`, after 3 untimed calls)."""
    import torch
    for _ in range(3):
        fn()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    for _ in range(steps):
        fn()
    ev[1].record(stream)
    torch.cuda.synchronize()
    return ev[0].elapsed_time(ev[1]) / steps


L2_BYTES = 126 << 20


def run_sweep(args):
    """Per-length throughput lines: the fused fast convolution, the phased
    Impl1op form (Fftm -> vmmul -> Fftm, three launches; benchmarks/fastconv.cpp
    :100-106) and the forward row Fftm, on three shapes: the reference
    benchmark's 64 rows x 2^4 .. 2^16 (benchmarks/fastconv.cpp:977-988), the
    256 x {256 .. 65536} row sweep, and a fixed 2^24-sample batch per length;
    then the 4096 x 4096 2-D FFT.  Kernel time by CUDA events.  The Fftm and
    2-D lines carry the forward transform's rel-L2 against FP64 (numpy) and the
    forward -> inverse round trip's rel-L2 against the input, on uniform
    [-1, 1] data."""
    import torch

    import openvsip_b200 as ov
    from openvsip_b200 import synth
    torch.cuda.set_device(0)
    peak, _ = measured_peak()
    stream = torch.cuda.current_stream()
    shapes = [("64 rows (reference benchmark shape)", 64, range(4, 17)), ("256 rows", 256, range(8, 17)),
              ("2^24 samples", None, range(8, 17))]
    for label, rows_fixed, logs in shapes:
        for logn in logs:
            n = 1 << logn
            rows = rows_fixed or (1 << 24) // n
            x = torch.randn(rows, n, dtype=torch.complex64, device="cuda")
            y = torch.empty_like(x)
            tmp = torch.empty_like(x)
            rep_np = np.exp(2j * np.pi * np.random.default_rng(logn).random(n)).astype(np.complex64)
            rep = torch.from_numpy(rep_np).cuda()
            if args.threads:
                for kind_id in (0, 2):
                    ov.lib().fcb_tune_set(n, kind_id, args.threads)
            fc = ov.Fastconv(rep_np, rows)
            fwd = ov.Fftm(rows, n, ov.fft_fwd)
            inv = ov.Fftm(rows, n, ov.fft_inv, 1.0 / n)

            def phased():
                fwd(x, tmp)
                ov.vmmul(rep, tmp, tmp)
                inv(tmp, y)

            # accuracy on up to 8 rows of uniform [-1, 1] data: the forward transform against FP64,
            # and the round trip forward -> inverse (scale 1/n) against the input
            u = torch.from_numpy(synth.sweep_matrix(logn, min(rows, 8), n)).cuda()
            fu = fwd(u)
            back = inv(fu)
            un = u.cpu().numpy()
            acc = {"fwd_rel_l2_vs_fp64": rel_l2(fu.cpu().numpy(), np.fft.fft(un.astype(np.complex128), axis=1)),
                   "roundtrip_rel_l2": rel_l2(back.cpu().numpy(), un)}
            for kind, fn, bps in (("fastconv", lambda: fc(x, y), 16.0), ("phased", phased, 48.0),
                                  ("fftm_fwd", lambda: fwd(x, y), 16.0)):
                steps = args.steps if rows * n >= (1 << 20) else max(args.steps, 2000)
                ms = _time_calls(fn, steps, stream)
                alg = bps * rows * n + (8.0 * n if kind != "fftm_fwd" else 0.0)
                gbs = alg / (ms / 1e3) / 1e9
                line = {"sweep": kind, "n": n, "rows": rows, "shape": label, "ms": ms,
                        "samples_per_s": rows * n / (ms / 1e3), "gbs": gbs, "frac": gbs / peak,
                        "alg_bytes_per_sample": bps, "l2_resident": 16 * rows * n < L2_BYTES,
                        "launches_per_call": 3 if kind == "phased" else 1,
                        "threads": fc.info()["threads"], "cluster": fc.info()["cluster_ctas"]}
                if kind == "fftm_fwd":
                    line.update(acc)
                print(json.dumps(line), flush=True)
            del fc, fwd, inv
    # 4096 x 4096 2-D FFT, forward and inverse (two HBM passes each: 32 B/sample), uniform [-1, 1]
    # data; round trip against the input and the forward transform against FP64
    x = torch.from_numpy(synth.sweep_matrix(4096, 4096, 4096)).cuda()
    y = torch.empty_like(x)
    f2, g2 = ov.Fft2d(4096, 4096, ov.fft_fwd), ov.Fft2d(4096, 4096, ov.fft_inv, 1.0 / 4096 ** 2)
    X = f2(x)
    xn = x.cpu().numpy()
    acc = {"fwd_rel_l2_vs_fp64": rel_l2(X.cpu().numpy(), np.fft.fft2(xn.astype(np.complex128))),
           "roundtrip_rel_l2": rel_l2(g2(X).cpu().numpy(), xn)}
    del X
    for name, plan in (("fft2d_fwd", f2), ("fft2d_inv", g2)):
        ms = _time_calls(lambda: plan(x, y), args.steps, stream)
        gbs = 32.0 * 4096 * 4096 / (ms / 1e3) / 1e9
        print(json.dumps({"sweep": name, "n": 4096, "rows": 4096, "shape": "4096 x 4096", "ms": ms,
                          "samples_per_s": 4096 * 4096 / (ms / 1e3), "gbs": gbs, "frac": gbs / peak, **acc}),
              flush=True)


def _cgauss_dev(rows, n, gen):
    import torch
    x = torch.randn(rows, n, 2, dtype=torch.float32, device="cuda", generator=gen)
    return torch.view_as_complex(x)  # sigma 1 per component


def fp64_fastconv(x, chirp64):
    """FP64 reference (numpy): ifft(fft(x) * conj(fft(chirp))) per row."""
    spec = np.conj(np.fft.fft(np.asarray(chirp64, dtype=np.complex128)))
    return np.fft.ifft(np.fft.fft(np.asarray(x, dtype=np.complex128), axis=1) * spec, axis=1)


BATCH_WORKLOAD = ("uneven batched fastconv, {jobs} jobs, pulses U{{16..512}}, samples from {{1024..32768}}, "
                  "own LFM replica per job (TBP U[50,1000]), complex Gaussian inputs")


def batch_block(args, world: int = 1, rank: int = 0, barrier=lambda: None) -> dict:
    """The uneven batch (512 jobs, pulses U{16..512}, samples from
    {1024..32768}, each job with its own LFM replica of TBP U[50, 1000],
    complex Gaussian inputs): one persistent graph-replayed launch per step on
    each rank.  With N ranks the jobs are partitioned by shard.partition_jobs
    (balanced by samples; large jobs cut into pulse ranges), so the block
    scales strongly.  Every job is checked against FP64 (numpy) on three of
    its rows (first, middle, last of each rank's piece).  The plain per-call
    GPU form (one fused Fastconv launch per job, plans made beforehand) is
    timed on the same data."""
    import torch

    from openvsip_b200 import autotune, shard, synth
    from openvsip_b200.batch import Batch
    from openvsip_b200.vsip import Fastconv
    sizes = tuple(int(v) for v in args.batch_sizes.split(",")) if args.batch_sizes else synth.SIZES
    jobs = synth.uneven_jobs(seed=3, njobs=args.batch_jobs, sizes=sizes)
    if world > 1:
        mine = shard.partition_jobs([(j["pulses"], j["n"]) for j in jobs], world)[rank]
    else:
        mine = [(i, 0, j["pulses"]) for i, j in enumerate(jobs)]
    gen = torch.Generator(device="cuda")
    xs, pieces = [], []
    for ji, b, e in mine:
        j = jobs[ji]
        gen.manual_seed(int(j["seed"]))
        xs.append(_cgauss_dev(j["pulses"], j["n"], gen)[b:e].contiguous())
        pieces.append((ji, b, e))
    ys = [torch.empty_like(x) for x in xs]
    chirps = [synth.job_replica(jobs[ji]).astype(np.complex64) for ji, _, _ in pieces]
    samples = sum(x.numel() for x in xs)

    def make(threads, order):
        bt = Batch(threads)
        ids = [bt.add_replica(c, kind="matched") for c in chirps]
        bt.set_jobs([(x, y, i) for x, y, i in zip(xs, ys, ids)], order=order)
        return bt

    if args.batch_threads:
        tune = {"threads": args.batch_threads, "order": "longest_first", "fixed": True}
    else:
        tune = autotune.tune_batch(make, reps=3)
    bt = make(tune["threads"], tune["order"])
    stream = torch.cuda.current_stream()
    bt.set_stream(stream.cuda_stream)
    for _ in range(args.warmup):
        bt.run()
    torch.cuda.synchronize()
    # accuracy of every job (3 rows each) against FP64
    errs = []
    for (ji, b, e), x, y, c in zip(pieces, xs, ys, chirps):
        rows = sorted({0, (e - b) // 2, e - b - 1})
        ref = fp64_fastconv(x[rows].cpu().numpy(), c)
        errs.append(rel_l2(y[rows].cpu().numpy(), ref))
    steps = max(3, min(args.steps, 20))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        t0.record(stream)
        for s_, e_ in ev:
            s_.record(stream)
            bt.run()
            e_.record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
    barrier()
    total_ms = shard.max_over_ranks(t0.elapsed_time(t1))
    ms = [s_.elapsed_time(e_) for s_, e_ in ev]
    mean = total_ms / steps
    all_samples = sum(j["pulses"] * j["n"] for j in jobs)
    alg = 16.0 * all_samples + 8.0 * sum(j["n"] for j in jobs)
    peak, peak_src = measured_peak()
    # the plain per-call GPU form: one fused launch per job, plans prepared beforehand
    plans = [Fastconv(c, x.shape[0], kind="matched") for c, x in zip(chirps, xs)]
    per_call_ms = shard.max_over_ranks(_time_calls(lambda: [p_(x, y) for p_, x, y in zip(plans, xs, ys)], 3, stream))
    n_plans = len(plans)
    del plans
    # and the phased Impl1op form per job (forward Fftm, vmmul<0>, inverse Fftm: three launches)
    from openvsip_b200.vsip import Fftm, fft_fwd, fft_inv, replica_spectrum, vmmul
    phased = [(Fftm(x.shape[0], x.shape[1], fft_fwd), Fftm(x.shape[0], x.shape[1], fft_inv, 1.0 / x.shape[1]),
               replica_spectrum(torch.from_numpy(c).cuda(), matched=True)) for c, x in zip(chirps, xs)]

    def run_phased():
        for (f, g, spec), x, y in zip(phased, xs, ys):
            f(x, y)
            vmmul(spec, y, y)
            g(y, y)

    phased_ms = shard.max_over_ranks(_time_calls(run_phased, 3, stream))
    del phased
    srt = sorted(ms)
    max_err = shard.max_over_ranks(max(errs))
    return {
        "workload": BATCH_WORKLOAD.format(jobs=len(jobs)) + (f" (row lengths {sizes} only)" if args.batch_sizes else ""),
        "samples_per_step": all_samples,
        "value": all_samples / (mean / 1e3), "unit": "complex samples/s", "ms_per_step": mean, "steps": steps,
        "scaling": "strong" if world > 1 else None,
        "latency_ms": {"p50": srt[len(srt) // 2], "p99": srt[min(len(srt) - 1, int(0.99 * len(srt)))]},
        "roofline": {"bound": "hbm", "achieved": alg / (mean / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (mean / 1e3) / 1e9 / peak, "peak_source": peak_src,
                     "alg_bytes_per_step": alg},
        "rel_l2_vs_fp64": {"max": max_err, "median_rank0": float(np.median(errs)), "jobs_checked": len(errs),
                           "rows_per_job": 3, "tolerance": 2e-6},
        "tuning": tune, "batch": bt.info(), "gpu_launches_per_step": 1,
        "per_call": {"ms": per_call_ms, "value": all_samples / (per_call_ms / 1e3), "launches_per_step": n_plans,
                     "how": "one fused Fastconv launch per job, plans prepared beforehand, device data"},
        "batch_over_per_call": per_call_ms / mean,
        "per_call_phased": {"ms": phased_ms, "value": all_samples / (phased_ms / 1e3), "launches_per_step": 3 * len(xs),
                            "how": "forward Fftm, vmmul<0>, inverse Fftm per job (the reference benchmark's Impl1op "
                                   "form), plans prepared beforehand, device data"},
        "batch_over_per_call_phased": phased_ms / mean, "clocks": clk.summary()}


def run_batch(args):
    """--batch: the uneven batch as a line of its own (not the headline)."""
    import torch
    torch.cuda.set_device(0)
    print(json.dumps(batch_block(args)), flush=True)


SERVE_WORKLOAD = ("served pulse compression, Poisson {rate:g} jobs/s for {seconds:g} s, uneven shapes, "
                  "64 resident replicas, 40 GB admission budget")


def serve_block(args) -> dict:
    """Served pulse-compression stream: Poisson arrivals at --serve-rate jobs/s
    for --serve-seconds, job shapes as in the uneven batch (pulses U{16..512},
    samples from {1024..32768}), 64 distinct replicas resident on the device,
    admission capped by a 40 GB device-memory budget.  Inputs are pre-staged on
    the device (a pool of complex Gaussian rows per length), so host<->device
    transfers are not part of the latency.  Every --serve-check-every-th job
    (default: every 8th) is checked against FP64: the FP64 results of the
    whole pool for every replica are computed on the host by numpy/scipy
    before the stream starts, and each job's output is compared with its rows
    on a separate CUDA stream while the stream runs."""
    import queue

    import scipy.fft
    import torch

    from openvsip_b200 import synth
    from openvsip_b200.serve import Server
    rng = np.random.default_rng(11)
    sizes = synth.SIZES
    replicas = []
    for i in range(64):
        n = sizes[i % len(sizes)]
        replicas.append(synth.lfm_chirp(n, float(rng.uniform(50, 1000)), n).astype(np.complex64))
    by_n = {n: [i for i, r in enumerate(replicas) if r.size == n] for n in sizes}
    gen = torch.Generator(device="cuda")
    gen.manual_seed(11)
    pool = {n: _cgauss_dev(512, n, gen) for n in sizes}
    torch.cuda.synchronize()
    # FP64 results of every pool row for every replica (host numpy/scipy, then resident on the device)
    cores = os.cpu_count() or 1
    refs, ref_cum = [], []
    pool_f = {n: scipy.fft.fft(pool[n].cpu().numpy().astype(np.complex128), axis=1, workers=cores) for n in sizes}
    for r in replicas:
        spec = np.conj(np.fft.fft(r.astype(np.complex128)))
        ref = scipy.fft.ifft(pool_f[r.size] * spec, axis=1, workers=cores)
        ref_cum.append(np.cumsum(np.sum(np.abs(ref) ** 2, axis=1)))
        refs.append(torch.from_numpy(ref).cuda())
    del pool_f
    torch.cuda.synchronize()
    rate, seconds = args.serve_rate, args.serve_seconds
    count = int(rng.poisson(rate * seconds))
    arrivals = np.sort(rng.uniform(0, seconds, count))
    shapes = [(int(rng.integers(16, 513)), int(sizes[int(rng.integers(0, len(sizes)))])) for _ in range(count)]
    rids = [by_n[n][int(rng.integers(0, len(by_n[n])))] for _, n in shapes]
    done_q = queue.Queue()
    lat, t_arrive = [], []
    every = max(1, int(args.serve_check_every))
    check_stream = torch.cuda.Stream()
    nums, dens = [], []

    def consume():
        # the client side: wait for each result in order; every `every`-th job
        # is compared with its FP64 rows on the check stream
        for i in range(count):
            r, p, n, rid = done_q.get()
            r.wait(timeout=600)
            lat.append(r.latency)
            t_arrive.append(r.t_submit)
            if i % every == 0:
                with torch.cuda.stream(check_stream):
                    d = r.out.to(torch.complex128) - refs[rid][:p]
                    nums.append(torch.linalg.vector_norm(d))
                dens.append(float(np.sqrt(ref_cum[rid][p - 1])))
                r.out.record_stream(check_stream)
            r.out = None

    consumer = threading.Thread(target=consume)
    with Server(replicas, memory_budget=40e9, slots=2) as srv:
        # warm-up (not timed): every length through both slots once, then a burst of
        # mixed jobs that fills large launches, and one check of each length, so module
        # loading and the allocators' first growth are not in the latencies
        warm = [srv.submit(pool[n][:512], by_n[n][0]) for n in sizes for _ in range(2)]
        warm += [srv.submit(pool[n][:p], by_n[n][0]) for p, n in shapes[:400]]
        for r in warm:
            r.wait(timeout=600)
        with torch.cuda.stream(check_stream):
            for n in sizes:
                torch.linalg.vector_norm(pool[n][:512].to(torch.complex128) - refs[by_n[n][0]][:512])
        check_stream.synchronize()
        del warm
        # keep the cyclic garbage collector out of the timed stream
        import gc
        gc.collect()
        gc.disable()
        consumer.start()
        t0 = time.perf_counter()
        with ClockSampler(torch.cuda.current_device()) as clk:
            for t_arr, (p, n), rid in zip(arrivals, shapes, rids):
                delay = t0 + t_arr - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                done_q.put((srv.submit(pool[n][:p], rid), p, n, rid))
            consumer.join()
        wall = time.perf_counter() - t0
        gc.enable()
        launches = srv.launches
        issue_ms = np.array(srv.issue_times) * 1e3
    check_stream.synchronize()
    errs = (torch.stack(nums).cpu().numpy() / np.array(dens)) if nums else np.array([np.nan])
    lat = np.array(lat) * 1e3
    samples = sum(p * n for p, n in shapes)
    # where in the stream the slow jobs were (arrival time in 10 s buckets)
    when = (np.array(t_arrive) - t0) // 10
    by_10s = {f"{int(k) * 10}-{int(k) * 10 + 10}s": round(float(np.percentile(lat[when == k], 99)), 3)
              for k in np.unique(when)}
    return {
        "workload": SERVE_WORKLOAD.format(rate=rate, seconds=seconds), "jobs": count, "launches": launches,
        "offered_samples_per_s": samples / seconds, "value": samples / wall, "unit": "complex samples/s",
        "wall_s": wall,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max()), "jobs_over_10ms": int((lat > 10).sum()),
                       "p99_by_arrival": by_10s},
        "rel_l2_vs_fp64": {"max": float(errs.max()), "median": float(np.median(errs)), "jobs_checked": int(errs.size),
                           "check_every": every, "tolerance": 2e-6,
                           "how": "FP64 numpy/scipy result of each job's rows, compared on a side CUDA stream"},
        "host_issue_ms_per_launch": {"p50": float(np.percentile(issue_ms, 50)),
                                     "p99": float(np.percentile(issue_ms, 99)), "max": float(issue_ms.max())},
        "clocks": clk.summary(),
        "inputs": "pre-staged on the device; latency is submit -> completion observed by the scheduler"}


def run_serve(args):
    """--serve: the served stream as a line of its own (not the headline)."""
    import torch
    torch.cuda.set_device(0)
    print(json.dumps(serve_block(args)), flush=True)


def phased_block(ov, x, y, chirp_dev, pulses, nsamp, steps, stream) -> dict:
    """The reference benchmark's Impl1op form (benchmarks/fastconv.cpp:100-106)
    on the GPU: forward Fftm, vmmul<0> by the replica spectrum, inverse Fftm
    scaled by 1/N -- three launches and three HBM round trips per step (48 B
    per sample of algorithmic traffic), on the same device data as the fused
    headline."""
    import torch
    spec = ov.replica_spectrum(chirp_dev, matched=True)
    tmp = torch.empty_like(y)
    fwd = ov.Fftm(pulses, nsamp, ov.fft_fwd)
    inv = ov.Fftm(pulses, nsamp, ov.fft_inv, 1.0 / nsamp)

    def step():
        fwd(x, tmp)
        ov.vmmul(spec, tmp, tmp)
        inv(tmp, y)

    ms = _time_calls(step, steps, stream)
    alg = 48.0 * pulses * nsamp + 8.0 * nsamp
    peak, _ = measured_peak()
    # Impl1ip: the same three steps in place on one buffer (benchmarks/fastconv.cpp, the in-place form)
    work = torch.empty_like(y)

    def step_ip():
        fwd(work, work)
        ov.vmmul(spec, work, work)
        inv(work, work)

    work.copy_(x)
    ms_ip = _time_calls(step_ip, steps, stream)
    return {"form": "Impl1op: Fftm(fwd) -> vmmul<0> -> Fftm(inv, 1/N), three launches per step",
            "value": pulses * nsamp / (ms / 1e3), "unit": "complex samples/s", "ms_per_step": ms, "steps": steps,
            "roofline": {"bound": "hbm", "alg_bytes_per_step": alg, "achieved": alg / (ms / 1e3) / 1e9,
                         "peak": peak, "unit": "GB/s", "frac": alg / (ms / 1e3) / 1e9 / peak},
            "gpu_launches_per_step": 3,
            "in_place": {"form": "Impl1ip: the same three launches in place on one buffer",
                         "value": pulses * nsamp / (ms_ip / 1e3), "ms_per_step": ms_ip,
                         "frac": alg / (ms_ip / 1e3) / 1e9 / peak}}


def matrix_block(ov, x, y, chirp, pulses, nsamp, steps, stream) -> dict:
    """The reference benchmark's matrix-of-coefficients form (Impl4mc,
    benchmarks/fastconv.cpp:857-969): inv_fftm(W * fwd_fftm(x)) with one
    replica spectrum per pulse, fused in one launch; the replica matrix is read
    once per step, so the algorithmic traffic is 24 B per sample."""
    import torch
    w = np.conj(np.fft.fft(chirp.astype(np.complex128)))[None, :] * np.exp(
        2j * np.pi * np.arange(pulses)[:, None] / pulses)          # a different spectrum per pulse
    fc = ov.Fastconv(w.astype(np.complex64), pulses)
    ms = _time_calls(lambda: fc(x, y), steps, stream)
    alg = 24.0 * pulses * nsamp
    peak, _ = measured_peak()
    ys = y[:8].cpu().numpy()
    ref = np.fft.ifft(np.fft.fft(x[:8].cpu().numpy().astype(np.complex128), axis=1) *
                      w[:8].astype(np.complex64).astype(np.complex128), axis=1)
    return {"form": "Impl4mc: inv_fftm(W * fwd_fftm(x)), one spectrum per pulse, one fused launch per step",
            "value": pulses * nsamp / (ms / 1e3), "unit": "complex samples/s", "ms_per_step": ms, "steps": steps,
            "roofline": {"bound": "hbm", "alg_bytes_per_step": alg, "achieved": alg / (ms / 1e3) / 1e9,
                         "peak": peak, "unit": "GB/s", "frac": alg / (ms / 1e3) / 1e9 / peak},
            "rel_l2_vs_fp64": rel_l2(ys, ref), "gpu_launches_per_step": 1}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="fcb", choices=["fcb", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="leave the uneven-batch block out of the line")
    ap.add_argument("--no-serve", action="store_true", help="leave the served-stream block out of the line")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--threads", type=int, default=0, help="force the 256- or 512-thread kernel variant")
    ap.add_argument("--sweep", action="store_true", help="per-length throughput lines instead of the benchmark")
    ap.add_argument("--batch", action="store_true", help="uneven batched workload line instead of the benchmark")
    ap.add_argument("--batch-jobs", type=int, default=512)
    ap.add_argument("--batch-sizes", default="",
                    help="comma-separated row lengths of the batch's jobs (profiling one length; default the mix)")
    ap.add_argument("--batch-threads", type=int, default=0,
                    help="batch kernel variant (256, 512 or -256) instead of the autotuned one")
    ap.add_argument("--serve", action="store_true", help="served-stream line instead of the benchmark")
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-check-every", type=int, default=8,
                    help="check every k-th served job against FP64 (checking all of them from the client thread "
                         "competes with the scheduler thread for the interpreter and inflates the latencies)")
    ap.add_argument("--pulses", type=int, default=PULSES, help="override the pulse count (profiling other shapes)")
    ap.add_argument("--samples", type=int, default=NSAMP, help="override the samples per pulse")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()
    if args.sweep:
        run_sweep(args)
        return
    if args.batch:
        run_batch(args)
        return
    if args.serve:
        run_serve(args)
        return

    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    import openvsip_b200 as ov
    from openvsip_b200 import shard, synth

    pulses, nsamp = args.pulses, args.samples
    default_shape = (pulses, nsamp) == (PULSES, NSAMP)
    if args.threads:
        ov.lib().fcb_tune_set(nsamp, 2, args.threads)
    job = synth.large_fastconv(seed=1000 + rank, pulses=pulses, n=nsamp, tbp=TBP, echoes=ECHOES)
    x_host = job["data"]
    chirp = job["chirp"].astype(np.complex64)
    # the replica spectrum is built by the library in FP64 on the GPU from the time-domain chirp
    # (replica kind "matched": conj(FFT(chirp)))
    fc = ov.Fastconv(chirp, pulses, kind="matched")
    info = fc.info()
    xin = [torch.from_numpy(x_host).cuda(), torch.from_numpy(np.roll(x_host, 1, axis=0)).cuda()]
    yout = torch.empty_like(xin[0])
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    for i in range(args.warmup):
        fc(xin[i % 2], yout)
    torch.cuda.synchronize()

    # accuracy of this run's output on a sample of rows (numpy FP64 FFT)
    fc(xin[0], yout)
    torch.cuda.synchronize()
    check_rows = min(32, pulses)
    ys = yout[:check_rows].cpu().numpy()
    ref = fp64_fastconv(x_host[:check_rows], chirp)
    rel = rel_l2(ys, ref)

    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    # throughput: K back-to-back launches between two events
    with ClockSampler(local) as clk:
        t_start.record(stream)
        for i in range(args.steps):
            fc(xin[i % 2], yout)
        t_end.record(stream)
        torch.cuda.synchronize()
    barrier()
    local_ms = t_start.elapsed_time(t_end)
    total_ms = shard.max_over_ranks(local_ms)  # max over ranks (NCCL all-reduce of one scalar)

    # per-launch latency (p50 / p99): a second pass with one event pair around each launch,
    # outside the throughput region so that its event records do not count there
    lat_steps = min(args.steps, 200)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(lat_steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(lat_steps)]
    for i in range(lat_steps):
        starts[i].record(stream)
        fc(xin[i % 2], yout)
        ends[i].record(stream)
    torch.cuda.synchronize()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]

    samples_step = pulses * nsamp
    value = samples_step * args.steps * world / (total_ms / 1e3)
    launch_ms = local_ms / args.steps  # average launch duration over the timed region
    alg_bytes = 16.0 * samples_step + 8.0 * nsamp
    achieved = alg_bytes / (launch_ms / 1e3) / 1e9
    peak, peak_src = measured_peak()

    # the phased Impl1op form on the same device data
    phased = phased_block(ov, xin[0], yout, torch.from_numpy(chirp).cuda(), pulses, nsamp, min(args.steps, 50),
                          stream)
    matrix = matrix_block(ov, xin[0], yout, chirp, pulses, nsamp, min(args.steps, 50), stream)

    # end to end through the public API with pinned host buffers: every step copies its input
    # in and its result out.  Streamed: the steps are submitted back to back (Fastconv.submit,
    # fcb_exec_async) and waited for once, so one step's copies in overlap the previous one's
    # last copies out; one call at a time (each waits for its result) is reported beside it.
    hin = torch.from_numpy(x_host).pin_memory().numpy()
    hout = torch.empty(x_host.shape, dtype=torch.complex64).pin_memory().numpy()
    fc(hin, hout)
    e2e_steps = min(args.steps, args.e2e_steps)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        fc(hin, hout)
    e2e_sync_s = time.perf_counter() - t0
    e2e_sync_value = samples_step * e2e_steps * world / shard.max_over_ranks(e2e_sync_s)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        fc.submit(hin, hout)
    fc.sync()
    e2e_s = time.perf_counter() - t0
    e2e_value = samples_step * e2e_steps * world / shard.max_over_ranks(e2e_s)
    # the same calls on pageable numpy arrays (how plain numpy callers and the plugin's
    # vsip::Matrix blocks arrive): staged through the plan's pinned buffers by host threads
    pout = np.empty_like(x_host)
    fc(x_host, pout)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        fc(x_host, pout)
    e2e_pg_s = time.perf_counter() - t0
    e2e_pg_value = samples_step * e2e_steps * world / shard.max_over_ranks(e2e_pg_s)
    del pout
    plugin = plugin_sample(pulses, nsamp, min(e2e_steps, 5)) if world == 1 else None

    # the served stream on one GPU (first: its latencies are the most sensitive to what ran
    # before), then the uneven batch on every rank (jobs partitioned across ranks)
    serve = None
    if world == 1 and not args.no_serve:
        import gc
        torch.cuda.synchronize()
        gc.collect()
        serve = serve_block(args)
        gc.collect()
        torch.cuda.empty_cache()
    batch = None if args.no_batch else batch_block(args, world, rank, barrier)

    if rank == 0:
        cpu = None
        standin = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_reference_sample(1) or cpu_port_sample()
            cpu.pop("seconds", None)
            cpu["host"] = host_info()
            standin = fftw_standin(x_host[:check_rows], np.conj(np.fft.fft(chirp.astype(np.complex128))).astype(
                np.complex64), ref)
        sorted_ms = sorted(step_ms)
        line = {
            "metric": baseline_metric(), "value": value, "unit": "complex samples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
            "data": "synthetic (seeded complex Gaussian + LFM echoes)",
            "config": {"workload": WORKLOAD if default_shape else WORKLOAD.replace(
                           f"{PULSES} pulses x {NSAMP} samples", f"{pulses} pulses x {nsamp} samples"),
                       "pulses": pulses, "samples": nsamp, "tbp": TBP,
                       "replica": "time-domain chirp, spectrum built by the library in FP64 on the GPU (matched)",
                       "parallelism": f"{world} independent batches (weak)",
                       "l2": f"inputs larger than L2 ({16 * samples_step >> 20} MB read+write per step, "
                             "2 alternating inputs)",
                       "kernel": {"threads": info["threads"], "cluster_ctas": info["cluster_ctas"],
                                  "smem_bytes": info["smem_bytes"],
                                  "variant": int(ov.lib().fcb_tune_get(nsamp, 2))}},
            "latency_ms": {"p50": sorted_ms[len(sorted_ms) // 2],
                           "p99": sorted_ms[min(len(sorted_ms) - 1, int(0.99 * len(sorted_ms)))],
                           "launches": lat_steps},
            "rel_l2_vs_fp64": rel,
            "rel_l2_rows_checked": check_rows,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": ncu_traffic() if default_shape else None,
                         "peak_source": peak_src,
                         "alg_bytes_per_launch": alg_bytes, "launch_ms": launch_ms},
            "cpu_baseline": cpu,
            "fftw_standin": standin,
            "e2e": {"value": e2e_value, "unit": "complex samples/s", "h2d_bytes_per_step": x_host.nbytes,
                    "d2h_bytes_per_step": x_host.nbytes, "steps": e2e_steps,
                    "how": "Fastconv.submit(host pinned in, host pinned out) per step, one sync at the end "
                           "(fcb_exec_async): chunked H2D / kernel / D2H on three streams, consecutive steps "
                           "overlapping on the PCIe link",
                    "one_call_at_a_time": {"value": e2e_sync_value, "unit": "complex samples/s",
                                           "how": "Fastconv(host pinned in, host pinned out), each call waits "
                                                  "for its result"},
                    "pageable": {"value": e2e_pg_value, "unit": "complex samples/s",
                                 "how": "Fastconv(numpy pageable in, numpy pageable out), each call waits for its "
                                        "result; chunks staged through pinned buffers by host threads"},
                    "plugin": plugin},
            "phased": phased,
            "matrix_of_coefficients": matrix,
            "batch": batch,
            "serve": serve,
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
