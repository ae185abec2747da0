"""Multi-GPU sharding of pulse-compression work: one process per GPU.

Rows (pulses) and jobs are independent, so the path shards with no exchange in
its data path.  The reference does the same: pulses are block-distributed with
a replicated replica (Map<Block_dist, Whole_dist>, benchmarks/fastconv.cpp:
54-65) and the FFT axis itself may not be distributed
(src/ovxx/signal/fft.hpp:404-414).  What crosses between ranks:

* each replica spectrum once, from one rank to all (broadcast_replica);
* the timing scalar, reduced to the maximum over ranks (max_over_ranks);
* results, only when a caller wants them on one rank (gather_rows).

Everything here runs on the process group the caller initialised (NCCL for
GPUs, gloo for CPU tests).
"""
from __future__ import annotations

import heapq

import numpy as np


def partition_rows(pulses: int, world: int) -> list[tuple[int, int]]:
    """Block distribution of `pulses` rows over `world` ranks: contiguous
    [begin, end) ranges whose sizes differ by at most one (Block_dist)."""
    if world < 1 or pulses < 0:
        raise ValueError("need world >= 1 and pulses >= 0")
    base, extra = divmod(pulses, world)
    out, b = [], 0
    for r in range(world):
        e = b + base + (1 if r < extra else 0)
        out.append((b, e))
        b = e
    return out


def partition_jobs(jobs, world: int) -> list[list[tuple[int, int, int]]]:
    """Assign jobs given as (pulses, samples) to ranks, balanced by samples.

    Returns per rank a list of (job index, row begin, row end).  Jobs are taken
    largest first and go to the least-loaded rank; a job larger than one
    rank's fair share is cut into pulse ranges first, so no rank waits on a
    single oversized job.  Every row of every job is assigned exactly once."""
    if world < 1:
        raise ValueError("need world >= 1")
    total = sum(p * n for p, n in jobs)
    fair = total / world if world else 0
    pieces = []
    for j, (p, n) in enumerate(jobs):
        if p <= 0:
            continue
        size = p * n
        k = max(1, min(p, int(np.ceil(size / fair)) if fair > 0 else 1))
        for b, e in partition_rows(p, k):
            if e > b:
                pieces.append(((e - b) * n, j, b, e))
    pieces.sort(key=lambda t: -t[0])
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for size, j, b, e in pieces:
        load, r = heapq.heappop(heap)
        out[r].append((j, b, e))
        heapq.heappush(heap, (load + size, r))
    for lst in out:
        lst.sort()
    return out


def _dist():
    import torch.distributed as dist
    return dist


def _device_for_backend():
    import torch
    dist = _dist()
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """Maximum of a per-rank scalar (e.g. the timed region's milliseconds)."""
    import torch
    dist = _dist()
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def broadcast_replica(replica, src: int = 0):
    """Send one complex64 replica (spectrum or time domain) from rank `src` to
    every rank, once; other ranks pass an array of the same shape (its
    contents are replaced).  Returns the numpy array on every rank."""
    import torch
    dist = _dist()
    arr = np.ascontiguousarray(replica, dtype=np.complex64)
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return arr
    t = torch.from_numpy(arr.view(np.float32).copy()).to(_device_for_backend())
    dist.broadcast(t, src=src)
    return t.cpu().numpy().view(np.complex64).reshape(arr.shape)


def gather_rows(local, parts: list[tuple[int, int]], dst: int = 0):
    """Collect each rank's rows (local: numpy complex64, rows of parts[rank])
    into the full matrix on rank `dst` (None elsewhere)."""
    import torch
    dist = _dist()
    local = np.ascontiguousarray(local, dtype=np.complex64)
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return local
    world, rank = dist.get_world_size(), dist.get_rank()
    cols = local.shape[1]
    rows_max = max(e - b for b, e in parts)
    dev = _device_for_backend()
    buf = np.zeros((rows_max, cols), dtype=np.complex64)
    buf[: local.shape[0]] = local
    t = torch.from_numpy(buf.view(np.float32)).to(dev)
    bufs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(bufs, t)
    if rank != dst:
        return None
    full = np.empty((parts[-1][1], cols), dtype=np.complex64)
    for r, (b, e) in enumerate(parts):
        full[b:e] = bufs[r].cpu().numpy().view(np.complex64)[: e - b]
    return full
