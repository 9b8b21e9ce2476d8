"""Strided passes fed by tensor copies (cp.async.bulk.tensor into shared memory).

With FB_FLAG_TMA the four-step column passes and strided axes whose lines
are neighbours in memory (FFTA's composite transform, src/algos.jl:51-118,
and the strided lines of fft_along_dim!, src/plan.jl:327-348) load whole
tiles of G lines with tensor copies, a tile ahead, instead of thread by
thread.  Only the way data reaches shared memory changes, so results must
equal the default thread-loaded kernels bit for bit and the FP64 oracle within
4 eps log2 N.
"""
import ctypes
import os

import numpy as np
import pytest

import ffta_b200 as F
from ffta_b200 import _lib

pytestmark = pytest.mark.gpu
NTHR = os.cpu_count() or 1


def _flag_clear():
    v = ctypes.c_int(0)
    assert _lib.lib.fb_kernel_error_flag(ctypes.byref(v), 1) == 0
    return v.value == 0


def _colmajor(shape, dt, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn(tuple(reversed(shape)), dtype=dt, device="cuda", generator=g)
    return x.permute(*reversed(range(len(shape))))


CASES = [
    # (dims in Julia order, region, dtype): four-step columns of long 1-D
    # transforms, and strided axes of 2-D / 3-D arrays
    ((2 ** 20, 4), 1, "c64"),
    ((2 ** 20, 2), 1, "c128"),
    ((2 ** 15, 8), 1, "c64"),
    ((512, 1536), 2, "c64"),
    ((1000, 1000), (1, 2), "c64"),
    ((1000, 1000), (1, 2), "c128"),
    ((512, 1024), 2, "c64"),
    ((96, 48, 40), (2, 3), "c128"),
]


@pytest.mark.parametrize("dims,region,kind", CASES)
def test_tensor_copies_equal_thread_loads(dims, region, kind):
    import torch
    import oracle
    dt = torch.complex64 if kind == "c64" else torch.complex128
    x = _colmajor(dims, dt, sum(dims))
    for planner in (F.plan_fft, F.plan_bfft):
        p = planner(x, region, _flags=F.FB_FLAG_TMA)
        q = planner(x, region)
        dp, dq = p.describe(x), q.describe(x)
        assert "<tma" in dp, dp
        assert "<tma" not in dq, dq
        a, b = p * x, q * x
        assert torch.equal(a, b), (dims, region, kind, dp)
        ref = oracle.fft_nd(x.cpu().numpy().astype(np.complex128), region, p.dir, prec="f64",
                            nthreads=NTHR)
        n = int(np.prod([dims[r - 1] for r in ([region] if isinstance(region, int) else region)]))
        eps = 2.0 ** -23 if kind == "c64" else 2.0 ** -52
        err = np.linalg.norm(a.cpu().numpy() - ref) / np.linalg.norm(ref)
        assert err <= 4 * eps * np.log2(n), (dims, err, dp)
    assert _flag_clear()


def test_unaligned_input_falls_back():
    """A view whose first element is not 16-byte aligned cannot be a tensor
    copy's base: the pass loads thread by thread and the result is the same."""
    import torch
    base = torch.randn(2 ** 15 * 4 + 1, dtype=torch.complex64, device="cuda")
    x = base[1:].view(4, 2 ** 15).T  # 8-byte offset
    y = torch.empty_like(x)  # same strides, aligned
    y.copy_(x)
    assert (x.data_ptr() % 16) != 0 and (y.data_ptr() % 16) == 0
    p = F.plan_fft(x, 1, _flags=F.FB_FLAG_TMA)
    assert "<tma" in p.describe(y)
    assert torch.equal(p * x, p * y)
    assert torch.equal(p * x, F.plan_fft(x, 1) * x)
    assert _flag_clear()
