"""bench.py's output contract.  The reference arm (CPU): one JSON line with the
metric, unit and direction of the GPU arm, the CPU baseline it measured and an
e2e block with no host-device traffic; ranks other than 0 print nothing.  The
GPU arm (on a B200): every key of its line, with consistent values."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_driver"))
                    and not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")),
                    reason="neither the reference build nor the oracle library is built")
def test_reference_arm_line():
    r = _run({}, "--steps", "1", "--warmup", "1")
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "complex samples/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert "metric" in line and "config" in line and "workload" in line["config"]


def test_reference_arm_other_ranks_print_nothing():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--steps", "1", "--warmup", "1")
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


@pytest.mark.gpu
def test_gpu_arm_line():
    # a short run of the GPU arm on a smaller shape: every key of the line, with sane values
    env = dict(os.environ)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--steps", "5", "--warmup", "3",
                        "--no-cpu-baseline", "--e2e-steps", "1", "--pulses", "64", "--batch-jobs", "8",
                        "--serve-seconds", "2", "--serve-rate", "100", "--serve-check-every", "1"],
                       capture_output=True, text=True, env=env, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e", "gpu_launches", "clocks"):
        assert k in line, k
    assert line["n_gpus"] == 1 and line["steps"] == 5 and line["warmup"] == 3 and line["gpu_launches"] == 5
    assert line["value"] > 0 and line["higher_is_better"] is True and line["scaling"] == "weak"
    roof = line["roofline"]
    assert roof["bound"] == "hbm" and roof["unit"] == "GB/s" and 0 < roof["frac"] == roof["achieved"] / roof["peak"]
    e2e = line["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] == e2e["d2h_bytes_per_step"] == 64 * 16384 * 8
    assert e2e["one_call_at_a_time"]["value"] > 0 and e2e["pageable"]["value"] > 0
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(line["clocks"])
    assert line["rel_l2_vs_fp64"] <= 2e-6
    ph = line["phased"]
    assert ph["value"] > 0 and ph["gpu_launches_per_step"] == 3 and ph["roofline"]["frac"] > 0
    assert ph["in_place"]["value"] > 0
    mc = line["matrix_of_coefficients"]
    assert mc["value"] > 0 and mc["rel_l2_vs_fp64"] <= 2e-6
    b = line["batch"]
    assert b["value"] > 0 and b["rel_l2_vs_fp64"]["max"] <= 2e-6 and b["rel_l2_vs_fp64"]["jobs_checked"] == 8
    assert b["per_call"]["launches_per_step"] == 8 and b["batch_over_per_call"] > 0
    assert b["per_call_phased"]["launches_per_step"] == 24 and b["batch_over_per_call_phased"] > 0
    sv = line["serve"]
    assert sv["jobs"] > 0 and sv["rel_l2_vs_fp64"]["jobs_checked"] == sv["jobs"]
    assert sv["rel_l2_vs_fp64"]["max"] <= 2e-6 and sv["latency_ms"]["p99"] >= sv["latency_ms"]["p50"] > 0
