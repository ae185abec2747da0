"""Batched uneven fast convolution (one persistent graph-replayed launch):
every job's result against the FP64 oracle (rel-L2 <= 2e-6), replay
determinism, in-place jobs, job order, and equality with the same job run alone
through the single-job path."""
import numpy as np
import pytest

from conftest import crandn, pinned_variant
from openvsip_b200 import Fastconv, synth
from openvsip_b200.batch import Batch

pytestmark = pytest.mark.gpu
RTOL = 2e-6


def _mix(seed, njobs, pulses=(16, 64), sizes=(256, 1024, 2048, 4096, 8192, 16384, 32768)):
    return synth.uneven_jobs(seed=seed, njobs=njobs, pulses=pulses, sizes=sizes)


@pytest.mark.parametrize("threads", [256, 512, -256])
def test_batch_uneven_jobs_vs_fp64(oracle, threads):
    import torch
    jobs = _mix(1, 20)
    b = Batch(threads)
    xs, ys, reps, jl = [], [], [], []
    for j in jobs:
        x = synth.job_data(j)
        chirp = synth.job_replica(j)
        rid = b.add_replica(chirp.astype(np.complex64), kind="matched")
        dx = torch.from_numpy(x).cuda()
        dy = torch.empty_like(dx)
        xs.append(x)
        ys.append(dy)
        reps.append(np.conj(np.fft.fft(chirp.astype(np.complex64).astype(np.complex128))).astype(np.complex64))
        jl.append((dx, dy, rid))
    b.set_jobs(jl)
    info = b.info()
    assert info["samples"] == sum(j["pulses"] * j["n"] for j in jobs)
    b.run()
    b.sync()
    first = [y.cpu().numpy() for y in ys]
    for x, y, r, j in zip(xs, first, reps, jobs):
        err = oracle.rel_l2(y, oracle.fastconv(x, r))
        assert err <= RTOL, (j, err)
    # graph replay gives the same result
    for y in ys:
        y.zero_()
    b.run()
    b.sync()
    for y0, y in zip(first, ys):
        np.testing.assert_array_equal(y.cpu().numpy(), y0)


# single-job variants with the same arithmetic as each batch kernel: the
# 256- and 512-thread kernels run 32 samples per thread at every length; the
# wide one runs 64 at 16384 and 32768
_SAME_ARITHMETIC = {512: {16384: 512, 32768: 512}, -256: {16384: -256, 32768: -256}}


@pytest.mark.parametrize("threads", [512, -256])
def test_batch_equals_single_job_path_and_order(oracle, threads):
    import torch
    jobs = _mix(2, 12, pulses=(3, 40))
    b = Batch(threads)
    jl, singles = [], []
    pins = _SAME_ARITHMETIC[threads]
    for j in jobs:
        x = synth.job_data(j)
        rep = crandn(np.random.default_rng(j["seed"]), (j["n"],))
        rid = b.add_replica(rep, kind="spectrum")
        dx = torch.from_numpy(x).cuda()
        jl.append((dx, torch.empty_like(dx), rid))
        with pinned_variant(16384, 2, pins[16384]), pinned_variant(32768, 2, pins[32768]):
            singles.append(Fastconv(rep, x.shape[0])(dx))
    b.set_jobs(jl, order="as_given")
    b.run()
    b.sync()
    for (dx, dy, _), s in zip(jl, singles):
        np.testing.assert_array_equal(dy.cpu().numpy(), s.cpu().numpy())
    # in place, longest-first order: same values
    jl2 = [(dx.clone(), None, rid) for dx, _, rid in jl]
    jl2 = [(x, x, rid) for x, _, rid in jl2]
    b.set_jobs(jl2)
    b.run()
    b.sync()
    for (x, _, _), s in zip(jl2, singles):
        np.testing.assert_array_equal(x.cpu().numpy(), s.cpu().numpy())


def test_batch_rejects_bad_jobs():
    import torch
    from openvsip_b200 import FcbError
    b = Batch()
    rid = b.add_replica(np.ones(1024, dtype=np.complex64))
    x = torch.zeros(4, 2048, dtype=torch.complex64, device="cuda")
    with pytest.raises(FcbError):
        b.set_jobs([(x, x, rid)])  # replica length != row length
    with pytest.raises(FcbError):
        b.add_replica(np.ones(65536, dtype=np.complex64))  # beyond the batch's 32768


@pytest.mark.parametrize("threads", [-256, 512])
def test_c3_full_config_every_job_vs_fp64(oracle, threads):
    """The full uneven batch: 512 jobs, pulses U{16..512}, samples from
    {1024..32768}, each job with its own LFM replica (TBP U[50, 1000]), about
    1.45 G samples in one persistent launch.  Every job is checked against the
    FP64 oracle on three seeded rows (first, a random one, last), after two
    replays of the graph (the second must be bit-identical to the first)."""
    import torch
    jobs = synth.uneven_jobs(seed=3, njobs=512)
    gen = torch.Generator(device="cuda")
    b = Batch(threads)
    xs, ys, chirps, jl = [], [], [], []
    for j in jobs:
        gen.manual_seed(int(j["seed"]))
        x = torch.view_as_complex(torch.randn(j["pulses"], j["n"], 2, device="cuda", generator=gen))
        chirp = synth.job_replica(j).astype(np.complex64)
        rid = b.add_replica(chirp, kind="matched")
        y = torch.full_like(x, float("nan"))
        xs.append(x)
        ys.append(y)
        chirps.append(chirp)
        jl.append((x, y, rid))
    b.set_jobs(jl)
    assert b.info()["samples"] == sum(j["pulses"] * j["n"] for j in jobs) > 1_000_000_000
    b.run()
    b.sync()
    rng = np.random.default_rng(3)
    picks = [sorted({0, int(rng.integers(0, j["pulses"])), j["pulses"] - 1}) for j in jobs]
    first = [y[r].cpu().numpy() for y, r in zip(ys, picks)]
    b.run()
    b.sync()
    worst = 0.0
    for k, (j, x, y, c, rows) in enumerate(zip(jobs, xs, ys, chirps, picks)):
        got = y[rows].cpu().numpy()
        np.testing.assert_array_equal(got, first[k])
        spec = np.conj(np.fft.fft(c.astype(np.complex128))).astype(np.complex64)
        want = oracle.fastconv(x[rows].cpu().numpy(), spec)
        err = oracle.rel_l2(got, want)
        worst = max(worst, err)
        assert err <= RTOL, f"job {k} ({j['pulses']} x {j['n']}): rel-L2 {err:.3e}"
    # no job row was left unwritten (NaN-filled outputs)
    assert all(bool(torch.isfinite(torch.view_as_real(y)).all()) for y in ys)


@pytest.mark.parametrize("threads", [512, -256])
def test_batch_more_jobs_than_the_shared_index(oracle, threads):
    # more than 1024 jobs: the unit -> job lookup runs on the job table in global
    # memory instead of its copy in shared memory; every job equals the
    # single-job path (the same arithmetic) and the first and last match FP64
    import torch
    rng = np.random.default_rng(1100)
    b = Batch(threads)
    n_list = [256, 512, 1024]
    reps = {n: crandn(rng, (n,)) for n in n_list}
    rids = {n: b.add_replica(reps[n], kind="spectrum") for n in n_list}
    jl, xs = [], []
    for k in range(1100):
        n = n_list[k % 3]
        x = crandn(rng, (1 + k % 3, n))
        dx = torch.from_numpy(x).cuda()
        jl.append((dx, torch.full_like(dx, float("nan")), rids[n]))
        xs.append(x)
    b.set_jobs(jl, order="as_given")
    b.run()
    b.sync()
    plans = {n: Fastconv(reps[n], 3) for n in n_list}
    for (dx, dy, _), x in zip(jl, xs):
        np.testing.assert_array_equal(dy.cpu().numpy(), plans[x.shape[1]](dx).cpu().numpy())
    for k in (0, 1099):
        n = xs[k].shape[1]
        assert oracle.rel_l2(jl[k][1].cpu().numpy(), oracle.fastconv(xs[k], reps[n])) <= RTOL
