"""Continuous-batching server: requests that arrive while others run are
admitted as launch slots and the memory budget free up, run batched with other
jobs, and each result is the same as the job run alone (same kernels), within
the 2e-6 relative-L2 tolerance against FP64."""
import numpy as np
import pytest

from conftest import pinned_variant
from openvsip_b200 import Fastconv, synth
from openvsip_b200.serve import Server

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone_results(oracle):
    import torch
    rng = np.random.default_rng(5)
    chirps = [synth.lfm_chirp(n, float(rng.uniform(50, 1000)), n).astype(np.complex64)
              for n in (1024, 4096, 16384, 32768)]
    jobs = []
    for i in range(48):
        k = int(rng.integers(0, len(chirps)))
        n = chirps[k].size
        p = int(rng.integers(1, 40))
        x = torch.view_as_complex(torch.randn(p, n, 2, device="cuda"))
        jobs.append((x, k))
    # the server's batch kernel is the wide one (64 samples per thread at 16384
    # and 32768, 32 below): the alone results use the single-job variants with
    # the same arithmetic
    with pinned_variant(16384, 2, -256), pinned_variant(32768, 2, -256):
        alone = [Fastconv(chirps[k], x.shape[0], kind="matched")(x) for x, k in jobs]
    torch.cuda.synchronize()
    # a small budget so that admission has to wait for memory to free up
    budget = 3 * max(2 * x.numel() * 8 for x, _ in jobs)
    with Server(chirps, memory_budget=budget, slots=2, max_jobs=8, threads=-256) as srv:
        reqs = [srv.submit(x, k) for x, k in jobs]
        outs = [r.wait(timeout=60) for r in reqs]
        assert srv.launches > 1 and srv.launches < len(jobs)  # batched, in several launches
        assert abs(srv._mem) < 1e-6
    for (x, k), y, a in zip(jobs, outs, alone):
        np.testing.assert_array_equal(y.cpu().numpy(), a.cpu().numpy())
    for (x, k), y in list(zip(jobs, outs))[:6]:
        spec = np.conj(np.fft.fft(chirps[k].astype(np.complex128))).astype(np.complex64)
        assert oracle.rel_l2(y.cpu().numpy(), oracle.fastconv(x.cpu().numpy(), spec)) <= 2e-6
    lat = [r.latency for r in reqs]
    assert all(l > 0 for l in lat)


def test_server_rejects_oversized_job():
    import torch
    chirp = synth.lfm_chirp(1024, 100.0, 1024).astype(np.complex64)
    with Server([chirp], memory_budget=1e6, slots=1) as srv:
        with pytest.raises(ValueError):
            srv.submit(torch.zeros(100, 1024, dtype=torch.complex64, device="cuda"), 0)
        with pytest.raises(ValueError):
            srv.submit(torch.zeros(1, 1024, dtype=torch.complex64, device="cuda"), 3)
