"""Split-BF16 tensor-core radix-16 stage (FB_FLAG_TENSOR_STAGE).

FFTA computes only in the element type; this optional stage computes the
first radix-16 stage of ComplexF32 programs on the tcgen05 tensor cores
(inputs and DFT matrix split into three BF16 terms, six products accumulated
in FP32).  Its error must match the FP32 path: checked against the FP64
oracle on the reference's transform shapes (batched 1-D columns as in
src/plan.jl:194-207, 2-D as in src/plan.jl:210-257).
"""
import ctypes
import os

import numpy as np
import pytest

import ffta_b200 as F
from ffta_b200 import _lib

NTHR = os.cpu_count() or 1


def _x(shape, seed, dt=None):
    import torch
    dt = dt or torch.complex64
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn(tuple(reversed(shape)), dtype=dt, device="cuda", generator=g)
    return x.permute(*reversed(range(len(shape))))  # column-major view


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _flag_clear():
    v = ctypes.c_int(0)
    assert _lib.lib.fb_kernel_error_flag(ctypes.byref(v), 1) == 0
    return v.value == 0


def _check(shape, region, seed, direction=-1):
    import oracle
    x = _x(shape, seed)
    mk = F.plan_fft if direction < 0 else F.plan_bfft
    p = mk(x, region)
    q = mk(x, region, _flags=F.FB_FLAG_TENSOR_STAGE)
    assert "<tc>" in q.describe(x), q.describe(x)
    ref = oracle.fft_nd(x.cpu().numpy().astype(np.complex128), region, direction, prec="f64",
                        nthreads=NTHR)
    e32 = _rel((p * x).cpu().numpy(), ref)
    etc = _rel((q * x).cpu().numpy(), ref)
    n = int(np.prod([shape[r - 1] for r in ([region] if isinstance(region, int) else region)]))
    assert etc <= 4 * 2.0 ** -23 * np.log2(n), (etc, e32)
    assert etc <= 1.5 * e32 + 1e-8, (etc, e32)  # matches the FP32 path
    assert _flag_clear()
    return etc, e32


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2048, 4096, 6144, 8192])
def test_direct_stage_matches_fp32(n):
    _check((n, 96), 1, n)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [4096, 2048])
def test_backward_and_scaled(n):
    _check((n, 40), 1, n + 1, direction=1)
    x = _x((n, 40), 5)
    q = F.plan_ifft(x, 1, _flags=F.FB_FLAG_TENSOR_STAGE)
    back = F.plan_fft(x, 1, _flags=F.FB_FLAG_TENSOR_STAGE) * x
    assert _rel((q * back).cpu().numpy(), x.cpu().numpy()) <= 1e-6


@pytest.mark.gpu
def test_tile_stage_four_step_and_2d():
    _check((1 << 20, 2), 1, 3)       # four-step passes on the tile kernel
    _check((4096, 1024), [1, 2], 4)  # rows (direct) and strided columns (tile)


@pytest.mark.gpu
def test_flag_leaves_other_paths_alone():
    import torch
    # ComplexF64 and lengths without a first radix-16 stage are unchanged, bit for bit
    for shape, dt in (((4096, 8), torch.complex128), ((2187, 8), torch.complex64),
                      ((1000, 8), torch.complex64)):
        x = _x(shape, 9, dt)
        a = F.plan_fft(x, 1) * x
        q = F.plan_fft(x, 1, _flags=F.FB_FLAG_TENSOR_STAGE)
        assert "<tc>" not in q.describe(x)
        assert torch.equal(q * x, a)
