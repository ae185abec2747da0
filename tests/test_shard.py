"""Multi-process host logic of the sharded path on CPU (gloo, world_size 2):
row and job partitioning, the one-time replica broadcast, the max-over-ranks
timing reduction used by bench.py, and gathering rows back to one rank.  Each
rank's share of a fast convolution is computed with numpy here (no GPU in this
suite); the GPU kernels themselves are covered by the -m gpu tests."""
import os
import socket

import numpy as np
import pytest

from openvsip_b200 import shard


def test_partition_rows_is_block_distribution():
    assert shard.partition_rows(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert shard.partition_rows(2, 4) == [(0, 1), (1, 2), (2, 2), (2, 2)]
    with pytest.raises(ValueError):
        shard.partition_rows(4, 0)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_jobs_covers_every_row_once_and_balances(world):
    rng = np.random.default_rng(world)
    jobs = [(int(rng.integers(16, 513)), int(2 ** rng.integers(10, 16))) for _ in range(200)]
    jobs.append((4096, 32768))  # one job larger than a fair share: split by pulse ranges
    parts = shard.partition_jobs(jobs, world)
    covered = [np.zeros(p, dtype=int) for p, _ in jobs]
    loads = []
    for lst in parts:
        load = 0
        for j, b, e in lst:
            covered[j][b:e] += 1
            load += (e - b) * jobs[j][1]
        loads.append(load)
    assert all((c == 1).all() for c in covered)
    total = sum(p * n for p, n in jobs)
    assert max(loads) <= total / world * 1.05 + max(n for _, n in jobs) * 512


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        pulses, n = 37, 256
        rng = np.random.default_rng(5)
        x = (rng.standard_normal((pulses, n)) + 1j * rng.standard_normal((pulses, n))).astype(np.complex64)
        # the replica exists on rank 0 only and is broadcast once
        rep = (np.exp(1j * np.arange(n) * 0.3) if rank == 0 else np.zeros(n)).astype(np.complex64)
        rep = shard.broadcast_replica(rep)
        parts = shard.partition_rows(pulses, world)
        b, e = parts[rank]
        mine = np.fft.ifft(np.fft.fft(x[b:e], axis=1) * rep, axis=1).astype(np.complex64)
        full = shard.gather_rows(mine, parts)
        slowest = shard.max_over_ranks(1.5 + rank)
        if rank == 0:
            np.save(os.path.join(out_dir, "full.npy"), full)
            np.save(os.path.join(out_dir, "rep.npy"), rep)
        np.save(os.path.join(out_dir, f"max{rank}.npy"), np.array([slowest]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo_broadcast_gather_and_max(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    n = 256
    rep = np.load(tmp_path / "rep.npy")
    np.testing.assert_array_equal(rep, np.exp(1j * np.arange(n) * 0.3).astype(np.complex64))
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((37, n)) + 1j * rng.standard_normal((37, n))).astype(np.complex64)
    want = np.fft.ifft(np.fft.fft(x, axis=1) * rep, axis=1).astype(np.complex64)
    np.testing.assert_array_equal(np.load(tmp_path / "full.npy"), want)
    for r in range(world):
        assert float(np.load(tmp_path / f"max{r}.npy")[0]) == 2.5


def test_single_process_helpers_without_a_group():
    a = np.arange(4, dtype=np.complex64)
    assert shard.max_over_ranks(3.0) == 3.0
    np.testing.assert_array_equal(shard.broadcast_replica(a), a)
    np.testing.assert_array_equal(shard.gather_rows(a.reshape(2, 2), [(0, 2)]), a.reshape(2, 2))
