"""Continuous-batching pulse-compression server on one GPU.

Requests (one fast-convolution job each: a CUDA complex64 tensor of
pulses x samples and the id of a resident replica) arrive at any time.  A
scheduler thread keeps up to `slots` persistent batch launches in flight on
separate CUDA streams.  Whenever a slot is free it admits every waiting request
that fits the device-memory budget (input + output bytes of admitted, unfinished
jobs), up to `max_jobs` per launch, and launches them together.  Requests that
arrive while other launches run join the next free slot, so their work
overlaps on the device with the work already there.  Replica spectra stay
resident on the device for the server's lifetime.

Each job computes inv_fftm(vmmul<0>(R, fwd_fftm(x))) / N exactly as the
single-job path does (the same kernels), so a job's result does not depend on
the mix it was batched with.  Latency is host wall time from submit() to the
moment the scheduler observes the job's launch complete.
"""
from __future__ import annotations

import collections
import threading
import time

from .batch import Batch


class Request:
    __slots__ = ("x", "replica", "out", "t_submit", "t_start", "t_done", "nbytes", "_done", "error", "ready")

    def __init__(self, x, replica: int, ready):
        self.x = x
        self.ready = ready  # event on the submitter's stream: x is complete
        self.replica = replica
        self.out = None
        self.t_submit = time.perf_counter()
        self.t_start = None
        self.t_done = None
        self.nbytes = 2 * x.numel() * x.element_size()
        self._done = threading.Event()
        self.error = None

    def wait(self, timeout: float | None = None):
        if not self._done.wait(timeout):
            raise TimeoutError("request not finished")
        if self.error:
            raise self.error
        return self.out

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class Server:
    """replicas: time-domain replicas (numpy complex64) made resident as
    matched-filter spectra (kind "matched"), or spectra with kind="spectrum"."""

    def __init__(self, replicas, memory_budget: float = 40e9, slots: int = 2, max_jobs: int = 256,
                 threads: int = 0, kind: str = "matched", reserve_bytes: float | None = None):
        import torch
        self.torch = torch
        self.budget = float(memory_budget)
        self.max_jobs = int(max_jobs)
        self.streams = [torch.cuda.Stream() for _ in range(slots)]
        # Result buffers are allocated on the slot streams.  Reserve one large
        # segment in each stream's pool of the caching allocator up front, so
        # that serving splits cached memory instead of growing the pool with
        # cudaMalloc (tens to hundreds of ms) while requests wait.
        reserve = min(self.budget, 8e9) / slots if reserve_bytes is None else float(reserve_bytes)
        for st in self.streams:
            with torch.cuda.stream(st):
                torch.empty(int(reserve) // 8, dtype=torch.complex64, device="cuda")
        torch.cuda.synchronize()
        self.batches = []
        # one spare 256-sample replica per batch, used only to size the job
        # tables below (its id follows the callers' replicas)
        import numpy as np
        spare = np.ones(256, dtype=np.complex64)
        dummy = torch.zeros(1, 256, dtype=torch.complex64, device="cuda")
        for st in self.streams:
            b = Batch(threads)
            ids = [b.add_replica(r, kind=kind) for r in replicas]
            assert ids == list(range(len(replicas)))
            sid = b.add_replica(spare, kind="spectrum")
            b.set_stream(st.cuda_stream)
            # size the job table for max_jobs now: growing it while serving frees the old
            # table, which synchronises the whole device and stalls the other slot
            b.set_jobs([(dummy, dummy, sid)] * self.max_jobs, direct=True)
            self.batches.append(b)
        torch.cuda.synchronize()
        self.nreplicas = len(replicas)
        self._pending = collections.deque()
        self._inflight = [None] * slots  # (requests, event) per slot
        self._mem = 0.0
        self._cv = threading.Condition()
        self._stop = False
        self.completed = 0
        self.launches = 0
        self.issue_times = []  # host seconds spent issuing each launch
        self.issue_parts = []  # (allocation, job table, launch) seconds and jobs, per launch
        self._events = [torch.cuda.Event() for _ in range(slots)]
        self._thread = threading.Thread(target=self._loop, name="fcb-serve", daemon=True)
        self._thread.start()

    # -- client side -------------------------------------------------------
    def submit(self, x, replica: int) -> Request:
        if not (0 <= replica < self.nreplicas):
            raise ValueError("unknown replica id")
        ready = self.torch.cuda.Event()
        ready.record()
        r = Request(x, replica, ready)
        if r.nbytes > self.budget:
            raise ValueError("job larger than the memory budget")
        with self._cv:
            self._pending.append(r)
            self._cv.notify()
        return r

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify()
        self._thread.join()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- scheduler ---------------------------------------------------------
    def _admit(self):
        """Pop the waiting requests that fit the memory budget (FIFO)."""
        batch = []
        while self._pending and len(batch) < self.max_jobs:
            r = self._pending[0]
            if self._mem + r.nbytes > self.budget:
                break
            self._pending.popleft()
            self._mem += r.nbytes
            batch.append(r)
        return batch

    def _loop(self):
        torch = self.torch
        while True:
            progressed = False
            # retire finished launches
            for s, fl in enumerate(self._inflight):
                if fl is not None and fl[1].query():
                    now = time.perf_counter()
                    with self._cv:
                        for r in fl[0]:
                            r.t_done = now
                            self._mem -= r.nbytes
                            r._done.set()
                        self.completed += len(fl[0])
                    self._inflight[s] = None
                    progressed = True
            # launch waiting work into free slots
            for s, fl in enumerate(self._inflight):
                if fl is not None:
                    continue
                with self._cv:
                    reqs = self._admit()
                if not reqs:
                    break
                t_issue = time.perf_counter()
                try:
                    with torch.cuda.stream(self.streams[s]):
                        for r in reqs:
                            self.streams[s].wait_event(r.ready)
                            r.out = torch.empty_like(r.x)
                            r.t_start = time.perf_counter()
                    t_alloc = time.perf_counter()
                    b = self.batches[s]
                    b.set_jobs([(r.x, r.out, r.replica) for r in reqs], direct=True)
                    t_set = time.perf_counter()
                    b.run()
                    ev = self._events[s]
                    ev.record(self.streams[s])
                    self._inflight[s] = (reqs, ev)
                    self.launches += 1
                    t_end = time.perf_counter()
                    self.issue_times.append(t_end - t_issue)
                    self.issue_parts.append((t_alloc - t_issue, t_set - t_alloc, t_end - t_set, len(reqs)))
                except Exception as e:  # report to the clients, keep serving
                    with self._cv:
                        for r in reqs:
                            r.error = e
                            self._mem -= r.nbytes
                            r._done.set()
                progressed = True
            with self._cv:
                if self._stop and not self._pending and all(f is None for f in self._inflight):
                    return
                if not progressed:
                    idle = all(f is None for f in self._inflight) and not self._pending
                    self._cv.wait(0.01 if idle else 0.00005)
