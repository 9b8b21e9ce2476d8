"""Host-side logic of the FFTA-mirroring API, checked without a GPU.

These are the argument checks FFTA performs before any arithmetic
(test/argument_checking.jl, src/plan.jl:157-285); they raise before the
C library is asked to compute anything.
"""
import numpy as np
import pytest

import ffta_b200 as F


def test_empty_input_dimension_mismatch():
    # test/onedim/complex_forward.jl:35-37, test/twodim/complex_forward.jl:45-47
    with pytest.raises(F.DimensionMismatch):
        F.fft(np.zeros(0))
    with pytest.raises(F.DimensionMismatch):
        F.bfft(np.zeros(0, np.complex128))
    with pytest.raises(F.DimensionMismatch):
        F.fft(np.zeros((0, 0)))


@pytest.mark.parametrize("sz", [(103,), (8, 11), (6, 24, 25)])
def test_plan_size(sz):
    # test/argument_checking.jl:110-118
    x = np.zeros(sz, np.complex128)
    p = F.plan_fft(x)
    assert p.size() == sz
    assert p.size(1 + len(sz)) == 1
    with pytest.raises(F.DomainError):
        p.size(0)
    with pytest.raises(F.DomainError):
        p.size(-1)


def test_plan_array_mismatch_1d():
    # test/argument_checking.jl:13-23
    x = np.random.default_rng(0).standard_normal(3).astype(np.complex128)
    xp = np.concatenate([x, [1]])
    with pytest.raises(F.DimensionMismatch):
        F.plan_fft(x) * xp
    with pytest.raises(F.DimensionMismatch):
        F.plan_bfft(x) * xp


@pytest.mark.parametrize("region", [1, 2])
def test_plan_array_mismatch_2d(region):
    # test/argument_checking.jl:31-48
    x = np.ones((3, 3), np.complex128)
    xp = np.ones((4, 4), np.complex128)
    with pytest.raises(F.DimensionMismatch):
        F.plan_fft(x, region) * xp
    with pytest.raises(F.DimensionMismatch):
        F.plan_fft(x) * xp


def test_region_outside_array():
    # test/argument_checking.jl:70-84
    xc3 = np.ones((3, 3, 3), np.complex128)
    invalid_p = F.plan_fft(np.ones((3,) * 5, np.complex128), range(3, 6))
    with pytest.raises(F.DimensionMismatch, match="Plan region is outside array dimensions."):
        invalid_p * xc3
    xc4 = np.ones((1, 5, 5, 5), np.complex128)
    with pytest.raises(F.DimensionMismatch, match="Plan region is outside array dimensions."):
        F.mul_(xc4, invalid_p, xc4)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_io_mismatch(N):
    # test/argument_checking.jl:87-108
    x = np.ones((3,) * N, np.complex128)
    y = np.ones((4,) * N, np.complex128)
    for region in range(1, N + 1):
        with pytest.raises(F.DimensionMismatch):
            F.mul_(y, F.plan_fft(x, region), x)
    with pytest.raises(F.DimensionMismatch):
        F.mul_(y, F.plan_fft(x), x)
    with pytest.raises(F.DimensionMismatch):
        F.mul_(y, F.plan_fft(x, list(range(1, N))), x)


@pytest.mark.parametrize("n", [3, 4, 5])
def test_mutated_regions(n):
    # test/argument_checking.jl:130-147
    x = np.ones((2,) * n, np.complex128)
    p1 = F.plan_fft(x, list(range(1, n)))
    p1.region.append(n)
    with pytest.raises(F.DimensionMismatch, match="Region is invalid."):
        p1 * x
    p2 = F.plan_fft(x, list(range(1, n)))
    p2.region[0:2] = [2, 1]
    with pytest.raises(F.DimensionMismatch, match="Region is invalid."):
        p2 * x


@pytest.mark.parametrize("dt", [np.float16, np.int32, np.int64, object, np.complex256])
def test_unsupported_element_types_raise(dt):
    # no CPU fallback: anything but ComplexF32/F64 (and Float32/F64) is rejected
    x = np.ones(8, dtype=dt)
    with pytest.raises(F.ArgumentError):
        F.fft(x)


def test_plan_is_typed():
    p = F.plan_fft(np.ones(8, np.complex64))
    with pytest.raises(F.ArgumentError):
        p * np.ones(8, np.complex128)


def test_ifft_scale_is_planned():
    p = F.plan_ifft(np.ones((4, 6), np.complex128))
    assert p.scale == pytest.approx(1 / 24)
    assert p.dir == F.FFT_BACKWARD
