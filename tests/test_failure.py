"""Failure detection without a GPU fault.

FFTA raises Julia exceptions and has nothing asynchronous that could stall.
Here two kinds of failure are made on purpose, in the forms that leave the
GPU usable:

* device side: the kernels that wait on their own asynchronous work (the
  bulk copies of the FB_FLAG_STREAM kernel, the tensor-core products of the
  FB_FLAG_TENSOR_STAGE kernels) are given a wait limit of 1 ns through
  fb_set_wait_limit, so an ordinary copy or product "takes too long".  The
  kernel must set the error flag to -1, drain what it has in flight and
  return; the next launch with the default limit must be correct.
* host side: the serving loop refuses a request larger than its budget, a
  non-positive length and a length without a schedule, lets a waiting request
  be cancelled, and still completes every other request correctly.
"""
import ctypes
import os

import numpy as np
import pytest

from ffta_b200 import _lib

NTHR = os.cpu_count() or 1


def _flag(reset=True):
    v = ctypes.c_int(0)
    assert _lib.lib.fb_kernel_error_flag(ctypes.byref(v), int(reset)) == 0, _lib.last_error()
    return v.value


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_wait_limit_setter_needs_no_device():
    assert _lib.lib.fb_set_wait_limit(5) == 0
    assert _lib.lib.fb_set_wait_limit(0) == 0  # back to the default


def _timeout_then_recover(flags, n, batch):
    import torch
    import ffta_b200 as F
    import oracle
    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.randn(batch, n, dtype=torch.complex64, device="cuda", generator=g).T
    p = F.plan_fft(x, 1, _flags=flags)
    ref = oracle.fft_batched(x.T.cpu().numpy().astype(np.complex128), -1, nthreads=NTHR)
    assert _flag() == 0
    try:
        assert _lib.lib.fb_set_wait_limit(1) == 0
        y = p * x
        torch.cuda.synchronize()  # the kernel returned: no hang, no fault
        assert _flag() == -1
    finally:
        _lib.lib.fb_set_wait_limit(0)
    y = p * x
    torch.cuda.synchronize()
    assert _flag() == 0
    assert _rel(y.T.cpu().numpy(), ref) <= 1e-6
    return p.describe(x)


@pytest.mark.gpu
def test_stream_kernel_wait_runs_out():
    import ffta_b200 as F
    d = _timeout_then_recover(F.FB_FLAG_STREAM, 4096, 2048)
    assert "<stream>" in d, d


@pytest.mark.gpu
def test_tensor_stage_wait_runs_out():
    import ffta_b200 as F
    d = _timeout_then_recover(F.FB_FLAG_TENSOR_STAGE, 4096, 512)
    assert "<tc>" in d, d


def _big_prime(lo):
    def isp(v):
        if v % 2 == 0:
            return False
        f = 3
        while f * f <= v:
            if v % f == 0:
                return False
            f += 2
        return True
    v = lo | 1
    while not isp(v):
        v += 2
    return v


@pytest.mark.gpu
def test_server_refusals_and_cancel():
    import torch
    import ffta_b200 as F
    import oracle
    h = ctypes.c_void_p()
    budget = 8e9
    assert _lib.lib.fb_server_create(ctypes.byref(h), float(budget), 2, 0) == 0, _lib.last_error()
    try:
        g = torch.Generator(device="cuda").manual_seed(3)
        specs = [(4096, 8), (1000, 16), (2048, 4)]  # requests that fit
        xs = [torch.randn(b, n, dtype=torch.complex64, device="cuda", generator=g)
              for n, b in specs]
        ys = [torch.full_like(x, float("nan")) for x in xs]
        tk = ctypes.c_int64()

        def submit(n, dtype, b, x, y):
            return _lib.lib.fb_server_submit(h, n, dtype, -1, b, ctypes.c_void_p(x.data_ptr()),
                                             ctypes.c_void_p(y.data_ptr()), ctypes.byref(tk))

        assert submit(4096, _lib.FB_C32, 8, xs[0], ys[0]) == 0
        first = tk.value
        # larger than the whole budget (17 GB of data): refused before any
        # plan is made or any data is touched, no ticket taken
        rc = submit(4096, _lib.FB_C32, 1 << 18, xs[0], ys[0])
        assert rc == _lib.FB_ERR_OUT_OF_MEMORY and "budget" in _lib.last_error()
        # non-positive length (FFTA: DimensionMismatch)
        assert submit(0, _lib.FB_C32, 1, xs[0], ys[0]) == _lib.FB_ERR_DIMENSION_MISMATCH
        # a prime whose Bluestein pad has no ComplexF64 schedule (4.3 GB of
        # data fits the budget): the plan build fails; the data pointers are
        # never touched
        p = _big_prime(1 << 27)
        rc = submit(p, _lib.FB_C64, 1, xs[0], ys[0])
        assert rc == _lib.FB_ERR_UNSUPPORTED, (rc, _lib.last_error())
        # a waiting request is withdrawn; a second cancel of it fails
        assert submit(1000, _lib.FB_C32, 16, xs[1], ys[1]) == 0
        cancelled = tk.value
        assert cancelled == first + 1  # the refusals took no ticket
        assert _lib.lib.fb_server_cancel(h, cancelled) == 0
        assert _lib.lib.fb_server_cancel(h, cancelled) == _lib.FB_ERR_ARGUMENT
        assert submit(2048, _lib.FB_C32, 4, xs[2], ys[2]) == 0
        last = tk.value
        assert _lib.lib.fb_server_wait(h) == 0, _lib.last_error()
        # a dispatched request can no longer be cancelled
        assert _lib.lib.fb_server_cancel(h, last) == _lib.FB_ERR_ARGUMENT
        tks = (ctypes.c_int64 * 16)()
        tms = (ctypes.c_double * 16)()
        cnt = ctypes.c_int64()
        assert _lib.lib.fb_server_poll(h, 16, tks, tms, ctypes.byref(cnt)) == 0
        assert sorted(tks[:cnt.value]) == [first, last]
        st = (ctypes.c_int64 * 9)()
        assert _lib.lib.fb_server_stats(h, st, 9) == 0
        assert st[0] == 3 and st[8] == 1  # three requests accepted, one cancelled
        torch.cuda.synchronize()
        assert torch.isnan(ys[1]).all()  # the cancelled request never ran
        for i in (0, 2):
            ref = oracle.fft_batched(xs[i].cpu().numpy().astype(np.complex128), -1,
                                     nthreads=NTHR)
            assert _rel(ys[i].cpu().numpy(), ref) <= 4 * 2.0 ** -23 * np.log2(specs[i][0])
        assert F  # the package stays importable after the refusals
    finally:
        _lib.lib.fb_server_destroy(h)
