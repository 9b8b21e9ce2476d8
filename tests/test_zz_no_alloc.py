"""The allocation-free entry point fb_execute_noalloc_c32, through the C ABI.

fb_execute_noalloc_c32 serves callers that cannot call cudaMalloc when they
transform (allocator callbacks, real-time loops that forbid allocation after
start-up, hosts that pass only data buffers): it runs the two-pass schedule
with its intermediate in a static device array.  Its results must match the
regular entry point (fb_plan_create + fb_execute) within the tolerance the
parity tests use, 4 * eps(Float32) * log2(n), on consecutive calls that reuse
the same static scratch, and match the FP64 oracle within the same bound.
The test buffers are allocated here by torch; the entry point itself
allocates nothing.

This file is named to be collected last, and it runs alone as well.
"""
import ctypes

import numpy as np
import pytest

from ffta_b200 import _lib

pytestmark = pytest.mark.gpu

EPS32 = 2.0 ** -23


def tol(n):
    return 4 * EPS32 * max(1.0, np.log2(n))


def regular(x, n, batch, direction):
    """The existing entry point on the same device input."""
    import torch
    y = torch.empty_like(x)
    h = ctypes.c_void_p()
    rc = _lib.lib.fb_plan_create(ctypes.byref(h), n, _lib.FB_C32, direction, batch, 1, n, 1, n,
                                 73, 0)
    assert rc == 0, _lib.last_error()
    stream = torch.cuda.current_stream().cuda_stream
    rc = _lib.lib.fb_execute(h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                             ctypes.c_void_p(stream))
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    _lib.lib.fb_plan_destroy(h)
    return y.cpu().numpy()


def noalloc(x, n, batch, direction):
    import torch
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream().cuda_stream
    rc = _lib.lib.fb_execute_noalloc_c32(ctypes.c_void_p(x.data_ptr()),
                                         ctypes.c_void_p(y.data_ptr()), n, batch, direction,
                                         ctypes.c_void_p(stream))
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    return y.cpu().numpy()


def relerr(a, b):
    a = a.astype(np.complex128)
    b = b.astype(np.complex128)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def device_input(rng, n, batch):
    import torch
    x = (rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))).astype(
        np.complex64)
    return torch.from_numpy(x).cuda()


def fp64_oracle(x, direction):
    """FFTA's algorithm in Float64 (the CPU restatement) on the same input."""
    import oracle
    return oracle.fft_batched(x.cpu().numpy().astype(np.complex128), direction)


# lengths whose balanced split leaves N1 = 1 (1, 2, 3, 5: an empty stage
# program on pass 1), pure powers of three and of five (each pass runs only
# radix-9/3 or radix-5 stages), and mixed 2^a 3^b 5^c lengths
SIZES = [(4096, 64), (2 ** 20, 2), (3 * 5 ** 4 * 2 ** 5, 3), (1, 7), (2, 5), (3, 5), (5, 5),
         (16384, 8), (3 ** 9, 100), (5 ** 6, 4)]


@pytest.mark.parametrize("n,batch", SIZES)
def test_two_calls_match_regular_entry_point(n, batch):
    rng = np.random.default_rng(n)
    # two calls in a row, each against the regular entry point and the oracle
    for direction in (-1, 1):
        x = device_input(rng, n, batch)
        a = noalloc(x, n, batch, direction)
        b = regular(x, n, batch, direction)
        assert relerr(a, b) <= tol(n), (n, batch, direction)
        assert relerr(a, fp64_oracle(x, direction)) <= tol(n), (n, batch, direction)


def test_in_place():
    """in == out: pass 1 has read the whole input before pass 2 writes."""
    import torch
    rng = np.random.default_rng(3)
    x = device_input(rng, 4096, 64)
    ref = fp64_oracle(x, -1)
    stream = torch.cuda.current_stream().cuda_stream
    p = ctypes.c_void_p(x.data_ptr())
    rc = _lib.lib.fb_execute_noalloc_c32(p, p, 4096, 64, -1, ctypes.c_void_p(stream))
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert relerr(x.cpu().numpy(), ref) <= tol(4096)


def test_consecutive_calls_of_different_sizes_share_the_scratch():
    rng = np.random.default_rng(7)
    x1 = device_input(rng, 27648 // 27 * 25, 8)  # 25600 = 2^10 * 5^2
    x2 = device_input(rng, 1000, 100)
    first = noalloc(x1, x1.shape[1], 8, -1)
    second = noalloc(x2, 1000, 100, -1)
    assert relerr(first, regular(x1, x1.shape[1], 8, -1)) <= tol(x1.shape[1])
    assert relerr(second, regular(x2, 1000, 100, -1)) <= tol(1000)


def test_limits_are_rejected_before_any_work():
    import torch
    x = torch.zeros(16, dtype=torch.complex64, device="cuda")
    p = ctypes.c_void_p(x.data_ptr())
    # beyond the static scratch: 2^22 complex values
    rc = _lib.lib.fb_execute_noalloc_c32(p, p, 2 ** 20, 8, -1, None)
    assert rc == _lib.FB_ERR_ARGUMENT and "static scratch" in _lib.last_error()
    # a length with a prime factor other than 2, 3, 5
    rc = _lib.lib.fb_execute_noalloc_c32(p, p, 7 * 16, 1, -1, None)
    assert rc == _lib.FB_ERR_UNSUPPORTED
    rc = _lib.lib.fb_execute_noalloc_c32(p, p, 0, 1, -1, None)
    assert rc == _lib.FB_ERR_DIMENSION_MISMATCH
    rc = _lib.lib.fb_execute_noalloc_c32(p, p, 16, -1, -1, None)
    assert rc == _lib.FB_ERR_ARGUMENT and "batch" in _lib.last_error()
