"""Persistent bulk-copy variant of the contiguous-line kernel.

The variant changes only how lines reach shared memory (cp.async.bulk with
an mbarrier per buffer, two buffers per block), not the arithmetic, so its
results must equal the one-line-per-block kernel's bit for bit and the
oracle's within the usual tolerance.  FB_FLAG_STREAM selects it.  Batched
lines are FFTA's `_mul_loop!` columns (src/plan.jl:194-207).
"""
import ctypes
import os

import numpy as np
import pytest

import ffta_b200 as F
from ffta_b200 import _lib

NTHR = os.cpu_count() or 1


def _cols(n, batch, dt, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randn(batch, n, dtype=dt, device="cuda", generator=g).T  # n x batch, column-major


def _flag_clear():
    v = ctypes.c_int(0)
    assert _lib.lib.fb_kernel_error_flag(ctypes.byref(v), 1) == 0
    return v.value == 0


@pytest.mark.gpu
@pytest.mark.parametrize("n", [512, 1000, 1024, 2048, 2187, 3072, 4096, 4608, 6561])
@pytest.mark.parametrize("kind", ["c64", "c128"])
@pytest.mark.parametrize("batch", [1, 7, 333, 2000])
def test_stream_equals_block_kernel(n, kind, batch):
    import torch
    dt = torch.complex64 if kind == "c64" else torch.complex128
    x = _cols(n, batch, dt, n + batch)
    p = F.plan_fft(x, 1, _flags=F.FB_FLAG_STREAM)
    q = F.plan_fft(x, 1)
    assert "<stream>" not in q.describe(x)
    assert torch.equal(p * x, q * x), (p.describe(x), q.describe(x))
    pb = F.plan_bfft(x, 1, _flags=F.FB_FLAG_STREAM)
    assert torch.equal(pb * x, F.plan_bfft(x, 1) * x)
    assert _flag_clear()


@pytest.mark.gpu
def test_stream_is_used_and_matches_oracle():
    import torch
    import oracle
    x = _cols(4096, 300, torch.complex64, 5)
    p = F.plan_fft(x, 1, _flags=F.FB_FLAG_STREAM)
    assert "<stream>" in p.describe(x)
    y = (p * x).cpu().numpy().T
    ref = oracle.fft_batched(x.T.cpu().numpy().astype(np.complex128), -1, nthreads=NTHR)
    err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    assert err <= 1e-6, err


@pytest.mark.gpu
def test_stream_unaligned_lines_fall_back():
    # lines starting 8 bytes off a 16-byte boundary go to the block kernel
    import torch
    base = torch.randn(4096 * 64 + 1, dtype=torch.complex64, device="cuda")
    x = base[1:].view(64, 4096).T
    p = F.plan_fft(x, 1, _flags=F.FB_FLAG_STREAM)
    assert torch.equal(p * x, F.plan_fft(x, 1) * x)
    assert _flag_clear()


@pytest.mark.gpu
def test_stream_in_place_and_scaled():
    import torch
    x = _cols(2048, 513, torch.complex64, 9)
    ref = F.plan_ifft(x, 1) * x
    y = x.clone()
    p = F.plan_ifft(y, 1, _flags=F.FB_FLAG_STREAM)
    F.mul_(y, p, y)
    assert torch.equal(y, ref)
