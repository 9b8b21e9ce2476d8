"""Real transforms (rfft / brfft / irfft), FFTA src/plan.jl:102-150, 390-583.

CPU tests: FFTA's argument checks for real plans (test/argument_checking.jl).
GPU tests: the reference's real-transform test cases (test/onedim/real_*.jl,
test/twodim/real_*.jl) through the C ABI, with the oracle (the complex FFT of
the real input, 113-bit) as the reference; `==` where FFTA's tests use it.
"""
import os

import numpy as np
import pytest

import ffta_b200 as F

NTHR = os.cpu_count() or 1


def tol(prec, n):
    eps = 2.0 ** -23 if prec == "f32" else 2.0 ** -52
    return 4 * eps * max(1.0, np.log2(max(n, 2)))


def relerr(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d else 1.0)


# ------------------------------------------------------------------- CPU
def test_only_1d_and_2d():
    # test/argument_checking.jl:4-10
    xr = np.zeros((2, 2, 2))
    with pytest.raises(F.ArgumentError, match="only supports 1D and 2D FFTs"):
        F.plan_rfft(xr, range(1, 4))
    with pytest.raises(F.ArgumentError, match="only supports 1D and 2D FFTs"):
        F.plan_brfft(xr.astype(complex), 2, range(1, 4))


def test_real_plan_direction_errors():
    # test/argument_checking.jl:27-28, 52-53, 66-67
    xr1 = np.random.default_rng(0).standard_normal(3)
    xc1 = xr1.astype(complex)
    with pytest.raises(F.ArgumentError, match="only FFT_BACKWARD supported for complex vectors"):
        F.plan_rfft(xr1) * xc1
    with pytest.raises(F.ArgumentError, match="only FFT_FORWARD supported for real vectors"):
        F.plan_brfft(xc1, 5) * xr1
    xr2 = np.zeros((3, 3))
    with pytest.raises(F.ArgumentError, match="only FFT_BACKWARD supported for complex arrays"):
        F.plan_rfft(xr2, 1) * xr2.astype(complex)
    with pytest.raises(F.ArgumentError, match="only FFT_FORWARD supported for real arrays"):
        F.plan_brfft(xr2.astype(complex), 5, [1, 2]) * xr2


def test_real_plan_size_mismatch():
    # test/argument_checking.jl:24-25
    xr1 = np.random.default_rng(1).standard_normal(3)
    with pytest.raises(F.DimensionMismatch):
        F.plan_rfft(xr1) * np.concatenate([xr1, [1.0]])
    yr = np.zeros(2, complex)
    with pytest.raises(F.DimensionMismatch):
        F.plan_brfft(yr, 3) * np.zeros(3, complex)


@pytest.mark.parametrize("sz", [(103,), (8, 11)])
def test_real_plan_size(sz):
    # test/argument_checking.jl:120-127
    p = F.plan_rfft(np.zeros(sz))
    assert p.size() == sz
    assert p.size(1 + len(sz)) == 1
    with pytest.raises(F.DomainError):
        p.size(0)


def test_empty_real():
    with pytest.raises(F.DimensionMismatch):
        F.rfft(np.zeros(0))
    with pytest.raises(F.DimensionMismatch):
        F.brfft(np.zeros(0, complex), 0)


# ------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("N", [8, 11, 15, 16, 27, 100])
def test_rfft_delta(N):
    # test/onedim/real_forward.jl:3-11
    x = np.ones(N)
    y = F.rfft(x)
    ref = np.zeros(N // 2 + 1, complex)
    ref[0] = N
    assert np.abs(y - ref).max() <= 1e-12
    assert np.array_equal(y, F.rfft(x.reshape(1, 1, N), 3).reshape(-1))
    assert np.array_equal(y, F.rfft(np.asfortranarray(x.reshape(N, 1)), 1).reshape(-1))


@pytest.mark.gpu
@pytest.mark.parametrize("N", [8, 11, 15, 16, 27, 100])
def test_brfft_delta(N):
    # test/onedim/real_backward.jl:3-14
    y = F.brfft(np.ones(N, complex), 2 * (N - 1))
    ref = np.zeros(2 * (N - 1))
    ref[0] = 2 * (N - 1)
    assert np.abs(y - ref).max() <= 1e-12
    assert np.isrealobj(y)


@pytest.mark.gpu
@pytest.mark.parametrize("n", list(range(1, 65)) + [4096, 5329, 2 ** 20])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_rfft_against_oracle_and_round_trip(n, prec):
    import oracle
    rng = np.random.default_rng(n)
    dt = np.float64 if prec == "f64" else np.float32
    x = rng.standard_normal(n).astype(dt)
    y = F.rfft(x)
    assert y.shape == (n // 2 + 1,)
    ref = oracle.fft(x.astype(np.complex128), prec="f128" if n < 6000 else "f64",
                     nthreads=NTHR)[: n // 2 + 1]
    assert relerr(y, ref) <= tol(prec, n)
    # test/onedim/real_backward.jl:16-24: irfft(rfft(x), n) ~ x
    z = F.irfft(y, n)
    assert z.shape == (n,) and np.isrealobj(z)
    assert relerr(z, x) <= 10 * tol(prec, n)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 5, 8, 13, 16, 33])
def test_real_batched_equals_per_slice(n):
    # test/onedim/real_forward.jl:26-32 and real_backward.jl:27-41 (`==`)
    rng = np.random.default_rng(n)
    x = np.asfortranarray(rng.standard_normal((n, n + 1, n + 2)))
    for r in (1, 2, 3):
        y = F.rfft(x, r)
        ref = np.apply_along_axis(lambda v: F.rfft(np.ascontiguousarray(v)), r - 1, x)
        assert np.array_equal(y, ref), r
        b = F.brfft(y, x.shape[r - 1], r)
        refb = np.apply_along_axis(lambda v: F.brfft(np.ascontiguousarray(v), x.shape[r - 1]),
                                   r - 1, y)
        assert np.array_equal(b, refb), r
        assert relerr(F.irfft(y, x.shape[r - 1], r), x) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("n", list(range(1, 65, 7)) + [64])
def test_rfft_2d(n):
    # test/twodim/real_forward.jl:16-27 and real_backward.jl:12-23
    import oracle
    for m in (n, n + 1):
        rng = np.random.default_rng(100 * m + n)
        X = np.asfortranarray(rng.standard_normal((m, n)))
        Y = F.rfft(X)
        assert Y.shape == (m // 2 + 1, n)
        ref = oracle.fft(X.astype(np.complex128), prec="f128")[: m // 2 + 1, :]
        assert relerr(Y, ref) <= tol("f64", m * n)
        assert relerr(F.irfft(Y, m), X) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("N", [8, 11, 15, 16, 27, 100])
def test_real_2d_delta_and_regions(N):
    # test/twodim/real_forward.jl:3-14, real_backward.jl:3-9
    y = F.rfft(np.ones((N, N)))
    ref = np.zeros((N // 2 + 1, N), complex)
    ref[0, 0] = N * N
    assert np.allclose(y, ref)
    b = F.brfft(np.ones((N, N), complex), 2 * (N - 1))
    refb = np.zeros((2 * (N - 1), N))
    refb[0, 0] = N * 2 * (N - 1)
    assert np.allclose(b, refb, atol=1e-10)
    x = np.asfortranarray(np.random.default_rng(N).standard_normal((N, N)))
    r = F.rfft(x)
    assert np.allclose(r, F.rfft(np.asfortranarray(x.reshape(1, N, N, order="F")), [2, 3])[0])
    assert np.allclose(r, F.rfft(np.asfortranarray(x.reshape(1, 1, N, N, 1, order="F")),
                                 [3, 4])[0, 0, :, :, 0])


@pytest.mark.gpu
def test_real_on_device_tensors():
    import torch
    import oracle
    rng = np.random.default_rng(3)
    x = rng.standard_normal((64, 1000)).astype(np.float32)  # rows: 64 length-1000 signals
    t = torch.from_numpy(x).cuda()
    y = F.rfft(t.T, 1).T.cpu().numpy()
    ref = oracle.fft_batched(x.astype(np.complex128), -1, nthreads=NTHR)[:, :501]
    assert relerr(y, ref) <= tol("f32", 1000)
    back = F.irfft(F.rfft(t.T, 1), 1000, 1).T.cpu().numpy()
    assert relerr(back, x) <= 10 * tol("f32", 1000)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [4, 6, 18, 64, 1000, 2048, 4096, 8192, 16384])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_half_length_path(n, prec):
    """Even lengths whose half has a specialised kernel take FFTA's
    half-length algorithm (src/plan.jl:398-442 rfft, :466-495 brfft): the
    real line read as n/2 complex values, one kernel at half length with the
    split fused in.  Checked against the oracle's complex transform of the
    real input, by round trip, and bitwise against the same transform of
    each column alone."""
    import torch
    import oracle
    dt = torch.float32 if prec == "f32" else torch.float64
    B = 7
    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.randn(B, n, dtype=dt, device="cuda", generator=g)  # columns of a Julia n x B
    p = F.plan_rfft(x.T, 1)
    assert "REAL-HALF" in p.describe((n, B)), p.describe((n, B))
    y = p * x.T
    ref = oracle.fft_batched(x.cpu().numpy().astype(np.complex128), -1,
                             nthreads=NTHR)[:, : n // 2 + 1]
    assert relerr(y.T.cpu().numpy(), ref) <= tol(prec, n)
    for b in (0, B - 1):
        assert torch.equal(y[:, b], F.rfft(x[b].clone()))
    pb = F.plan_brfft(y, n, 1)
    assert "REAL-HALF" in pb.describe((n, B))
    z = F.irfft(y, n, 1)
    assert relerr(z.T.cpu().numpy(), x.cpu().numpy()) <= 10 * tol(prec, n)
    zb = pb * y
    refb = n * x.cpu().numpy()
    assert relerr(zb.T.cpu().numpy(), refb) <= 10 * tol(prec, n)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,r", [((6, 64, 5), 2), ((3, 4, 2048), 3), ((16, 32), 2)])
def test_half_length_strided_region(shape, r):
    """A single strided region dim takes the same half-length kernel (its
    lines copied to the front and back), so it equals the transform of each
    slice alone bit for bit, as FFTA's mapslices does (src/plan.jl:507-527)."""
    import oracle
    rng = np.random.default_rng(sum(shape))
    x = np.asfortranarray(rng.standard_normal(shape).astype(np.float32))
    n = shape[r - 1]
    p = F.plan_rfft(x, r)
    assert "REAL-HALF" in p.describe(shape) and "strided" in p.describe(shape)
    y = F.rfft(x, r)
    refs = np.apply_along_axis(lambda v: F.rfft(np.ascontiguousarray(v)), r - 1, x)
    assert np.array_equal(y, refs)
    ref = oracle.fft(x.astype(np.complex128), r, nthreads=NTHR)
    ref = np.take(ref, range(n // 2 + 1), axis=r - 1)
    assert relerr(y, ref) <= tol("f32", n)
    b = F.brfft(y, n, r)
    refb = np.apply_along_axis(lambda v: F.brfft(np.ascontiguousarray(v), n), r - 1, y)
    assert np.array_equal(b, refb)
    assert relerr(F.irfft(y, n, r), x) <= 10 * tol("f32", n)
