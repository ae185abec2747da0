"""The host-buffer path (numpy in, numpy out) on shapes large enough that rows
stream through the device in many chunks (ramped at both ends of a waiting
call; twice as large, with no ramp, for queued calls): results must be
identical to the device-pointer path (the same kernels per row) and match FP64
on sampled rows (relative L2 <= 2e-6)."""
import numpy as np
import pytest

from conftest import crandn
from openvsip_b200 import Fastconv, Fftm, fft_fwd

pytestmark = pytest.mark.gpu
RTOL = 2e-6


def _device(plan, x):
    import torch
    y = plan(torch.from_numpy(np.ascontiguousarray(x)).cuda())
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.mark.parametrize("rows,n", [(600, 16384), (6000, 1024), (300, 32768)])
def test_fastconv_host_chunks_equal_device(oracle, rows, n):
    rng = np.random.default_rng(rows + n)
    x = crandn(rng, (rows, n))
    rep = crandn(rng, (n,))
    fc = Fastconv(rep, rows)
    host = fc(x)
    np.testing.assert_array_equal(host, _device(fc, x))
    for r in (0, rows // 2, rows - 1):
        assert oracle.rel_l2(host[r:r + 1], oracle.fastconv(x[r:r + 1], rep)) <= RTOL


def test_fftm_host_chunks_strided_rows(oracle):
    rows, n = 700, 16384
    rng = np.random.default_rng(11)
    big = crandn(rng, (rows, n + 16))
    x = big[:, 8:n + 8]  # row stride n + 16: pitched copies
    f = Fftm(rows, n, fft_fwd, 0.5)
    out = np.zeros((rows, n + 4), dtype=np.complex64)
    f(x, out[:, 2:n + 2])
    np.testing.assert_array_equal(out[:, 2:n + 2], _device(f, x))
    assert not out[:, :2].any() and not out[:, -2:].any()
    for r in (0, 351, rows - 1):
        assert oracle.rel_l2(out[r:r + 1, 2:n + 2], 0.5 * oracle.fft_rows(x[r:r + 1], -1)) <= RTOL


def test_host_calls_back_to_back_and_in_place():
    # consecutive host calls reuse the staging buffers and streams of the plan
    rows, n = 400, 16384
    rng = np.random.default_rng(12)
    rep = crandn(rng, (n,))
    fc = Fastconv(rep, rows)
    xs = [crandn(rng, (rows, n)) for _ in range(3)]
    outs = [fc(x) for x in xs]
    for x, y in zip(xs, outs):
        np.testing.assert_array_equal(y, _device(fc, x))
    inplace = xs[0].copy()
    fc.in_place(inplace)
    np.testing.assert_array_equal(inplace, outs[0])


@pytest.mark.parametrize("rows,n,steps", [(600, 16384, 4), (1000, 2048, 3), (50, 1000, 3)])
def test_submitted_host_calls_equal_single_calls(oracle, rows, n, steps):
    # calls queued back to back with submit() (fcb_exec_async) reuse the plan's
    # staging buffers while earlier calls still drain: every step's output must
    # equal its own synchronous call's, bit for bit (n = 1000: Bluestein rows)
    import torch
    rng = np.random.default_rng(rows * n + steps)
    rep = crandn(rng, (n,))
    fc = Fastconv(rep, rows)
    xs = [torch.from_numpy(crandn(rng, (rows, n))).pin_memory().numpy() for _ in range(steps)]
    ys = [torch.empty((rows, n), dtype=torch.complex64).pin_memory().numpy() for _ in range(steps)]
    for x, y in zip(xs, ys):
        fc.submit(x, y)
    fc.sync()
    for x, y in zip(xs, ys):
        np.testing.assert_array_equal(y, fc(x))
    r = rows // 3
    assert oracle.rel_l2(ys[-1][r:r + 1], oracle.fastconv(xs[-1][r:r + 1], rep)) <= RTOL
    # one output buffer reused by every step (the last step's result stays)
    out = torch.empty((rows, n), dtype=torch.complex64).pin_memory().numpy()
    for x in xs:
        fc.submit(x, out)
    fc.sync()
    np.testing.assert_array_equal(out, fc(xs[-1]))


def test_waiting_and_queued_calls_interleaved():
    # a waiting call first (staging sized for its chunks), then queued calls
    # (chunks twice as large: the staging grows), a waiting call between queued
    # ones, and queued calls again: every output equals the device path's
    import torch
    rows, n = 900, 16384
    rng = np.random.default_rng(77)
    rep = crandn(rng, (n,))
    fc = Fastconv(rep, rows)
    xs = [torch.from_numpy(crandn(rng, (rows, n))).pin_memory().numpy() for _ in range(4)]
    want = [_device(fc, x) for x in xs]
    ys = [torch.empty((rows, n), dtype=torch.complex64).pin_memory().numpy() for _ in range(4)]
    np.testing.assert_array_equal(fc(xs[0]), want[0])
    fc.submit(xs[1], ys[1])
    fc.submit(xs[2], ys[2])
    np.testing.assert_array_equal(fc(xs[3]), want[3])
    fc.submit(xs[0], ys[0])
    fc.submit(xs[3], ys[3])
    fc.sync()
    for y, w in zip(ys, want):
        np.testing.assert_array_equal(y, w)


@pytest.mark.parametrize("pin_in,pin_out", [(False, False), (True, False), (False, True)])
def test_pageable_host_buffers_staged(oracle, pin_in, pin_out):
    # pageable sides go through the plan's pinned buffers and the copy threads
    # (ragged last chunk, strided rows on the pageable side), waiting and
    # queued calls alike
    import torch
    rows, n = 1100, 8192
    rng = np.random.default_rng(int(pin_in) * 2 + int(pin_out))
    rep = crandn(rng, (n,))
    fc = Fastconv(rep, rows)
    x = crandn(rng, (rows, n))
    want = _device(fc, x)

    def buf(pinned, like):
        if pinned:
            b = torch.empty(like.shape, dtype=torch.complex64).pin_memory().numpy()
            b[...] = like
            return b
        wide = np.zeros((like.shape[0], like.shape[1] + 8), dtype=np.complex64)
        wide[:, 4:4 + like.shape[1]] = like
        return wide[:, 4:4 + like.shape[1]]  # row stride n + 8

    xin = buf(pin_in, x)
    out = buf(pin_out, np.zeros_like(x))
    fc(xin, out)
    np.testing.assert_array_equal(out, want)
    out[...] = 0
    fc.submit(xin, out)
    fc.sync()
    np.testing.assert_array_equal(out, want)
    if not pin_out:
        assert not out.base[:, :4].any() and not out.base[:, -4:].any()
    r = rows - 1
    assert oracle.rel_l2(out[r:r + 1], oracle.fastconv(x[r:r + 1], rep)) <= RTOL


def test_pageable_calls_from_several_threads():
    # host threads with plans of their own share the copy threads: every
    # result equals the device path's
    import threading
    rng = np.random.default_rng(5)
    shapes = [(700, 16384), (3000, 2048), (900, 4096)]
    plans, xs, wants, outs, errs = [], [], [], [None] * 3, []
    for rows, n in shapes:
        fc = Fastconv(crandn(rng, (n,)), rows)
        x = crandn(rng, (rows, n))
        plans.append(fc)
        xs.append(x)
        wants.append(_device(fc, x))

    def work(i):
        try:
            for _ in range(3):
                outs[i] = plans[i](xs[i])
        except Exception as e:  # pragma: no cover - reported below
            errs.append(e)

    ts = [threading.Thread(target=work, args=(i,)) for i in range(3)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errs
    for o, w in zip(outs, wants):
        np.testing.assert_array_equal(o, w)
