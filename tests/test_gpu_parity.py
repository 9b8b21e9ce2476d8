"""GPU parity: the sm_100a library (through its C ABI) against the oracle.

Tolerances.  Each result is compared with an FP64-or-better oracle (the
__float128 run of the FFTA restatement for small N, its FP64 run for large N,
or the 50-digit golden DFTs) by relative L2 error, and must stay within
4 * eps(T) * log2(N) of the working precision T (eps(Float32) = 2^-23,
eps(Float64) = 2^-52; log2(N) taken as at least 1).  ComplexF32 N=4096
batches must also reach rel-L2 <= 1e-6.  Where FFTA's tests compare with `==`
(batched or strided transforms against the same transform of a contiguous
slice) the comparison here is bitwise as well.
"""
import os

import numpy as np
import pytest

import ffta_b200 as F
import oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "dft_golden.npz"))
NTHR = os.cpu_count() or 1
EPS = {np.complex64: 2.0 ** -23, np.complex128: 2.0 ** -52}


def tol(dtype, n):
    return 4 * EPS[np.dtype(dtype).type] * max(1.0, np.log2(max(n, 2)))


def relerr(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d else 1.0)


def crandn(rng, shape, dtype=np.complex128):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


def to_dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def dev_fft(x, region=None, direction=-1, **kw):
    """Run on device memory (fb_execute) and return a host array."""
    import torch
    t = to_dev(x)
    f = F.fft if direction == -1 else F.bfft
    y = f(t, region, **kw)
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.fixture(autouse=True, scope="module")
def _check_kernel_flag():
    yield
    v = __import__("ctypes").c_int()
    F._lib.lib.fb_kernel_error_flag(__import__("ctypes").byref(v), 1)
    assert v.value == 0, f"a kernel named radix {v.value} without a butterfly"


# ------------------------------------------------------------ golden vectors
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("n", [int(s) for s in GOLD["sizes"]])
def test_golden(n, dtype):
    x = GOLD[f"x_{n}"].astype(dtype)
    for direction, key in ((-1, "fwd"), (1, "bwd")):
        ref = GOLD[f"{key}_{n}"]
        # the golden input rounded to dtype: compare against the oracle on that input
        ref_rounded = oracle.fft_nd(x, None, direction, prec="f128")
        y = dev_fft(x, None, direction)
        assert relerr(y, ref_rounded) <= tol(dtype, n), (n, key)
        if dtype == np.complex128:
            assert relerr(y, ref) <= tol(dtype, n), (n, key)


# ------------------------------------------------------- reference test cases
@pytest.mark.parametrize("N", [8, 11, 15, 16, 27, 100, 275])
def test_delta_forward(N):
    # test/onedim/complex_forward.jl:3-11
    x = np.ones(N, np.complex128)
    y = F.fft(x)
    ref = np.zeros(N, complex)
    ref[0] = N
    assert np.abs(y - ref).max() <= 1e-12
    assert np.array_equal(y, F.fft(x.reshape(1, 1, N), 3).reshape(N))
    assert np.array_equal(y, F.fft(np.asfortranarray(x.reshape(N, 1)), 1).reshape(N))


@pytest.mark.parametrize("N", [8, 11, 15, 16, 27, 100, 103])
def test_delta_backward(N):
    # test/onedim/complex_backward.jl:4-11
    y = F.bfft(np.ones(N, np.complex128))
    ref = np.zeros(N, complex)
    ref[0] = N
    assert np.abs(y - ref).max() <= 1e-12


@pytest.mark.parametrize("n", list(range(1, 65)) + [73 * 73])
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_1d_against_oracle(n, dtype):
    # test/onedim/complex_forward.jl:14-24: the naive DFT (here the 113-bit oracle)
    rng = np.random.default_rng(n)
    x = crandn(rng, n, dtype)
    for direction in (-1, 1):
        ref = oracle.fft_nd(x, None, direction, prec="f128")
        assert relerr(dev_fft(x, None, direction), ref) <= tol(dtype, n), (n, direction)
        # host-array path (fb_execute_host) gives the same bits
        host = (F.fft if direction == -1 else F.bfft)(x)
        assert np.array_equal(host, dev_fft(x, None, direction))


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 64, 100, 1009])
def test_round_trip(n):
    # test/onedim/complex_backward.jl:13-20
    rng = np.random.default_rng(n)
    x = crandn(rng, n)
    y = F.fft(x)
    assert relerr(F.ifft(y), x) <= np.sqrt(np.finfo(float).eps)


@pytest.mark.parametrize("n", [1, 2, 5, 8, 13, 16, 31, 47, 64])
@pytest.mark.parametrize("direction", [-1, 1])
def test_batched_equals_per_slice(n, direction):
    # test/onedim/complex_forward.jl:26-32 (`==`): fft(x, r) == mapslices(fft, x; dims=r)
    rng = np.random.default_rng(n)
    x = np.asfortranarray(crandn(rng, (n, n + 1, n + 2)))
    f = F.fft if direction == -1 else F.bfft
    for r in (1, 2, 3):
        y = f(x, r)
        lines = np.ascontiguousarray(np.moveaxis(x, r - 1, -1)).reshape(-1, x.shape[r - 1])
        ref = f(lines.T.copy(order="F"), 1).T.reshape(np.moveaxis(x, r - 1, -1).shape)
        assert np.array_equal(np.moveaxis(y, r - 1, -1), ref), r
        one = f(np.ascontiguousarray(np.moveaxis(x, r - 1, -1)[1 % x.shape[0], 0]))
        assert np.array_equal(np.moveaxis(y, r - 1, -1)[1 % x.shape[0], 0], one)


# (N, bound) of test/onedim/accuracy.jl:15-43
POW2 = [(1 << 4, 3.0), (1 << 5, 3.0), (1 << 6, 3.0), (1 << 7, 3.0), (1 << 8, 4.0), (1 << 9, 4.0),
        (1 << 10, 8.0), (1 << 11, 8.0), (1 << 12, 10.0), (1 << 13, 12.0), (1 << 14, 14.0),
        (1 << 15, 20.0), (1 << 16, 22.0), (1 << 17, 28.0), (1 << 18, 28.0)]
POW3 = [(3, 3.0), (9, 3.0), (27, 3.0), (81, 4.0), (243, 5.0), (729, 7.0), (2187, 10.0),
        (6561, 13.0), (19683, 18.0)]


@pytest.mark.parametrize("N,bound", POW2 + POW3)
def test_twiddle_accuracy_bounds(N, bound):
    # worst over 5 seeds of ||fft(x32) - F32(fft(F64(x32)))|| / ||.|| / eps(Float32)
    worst = 0.0
    for seed in range(1, 6):
        rng = np.random.default_rng(seed)
        x32 = crandn(rng, N, np.complex64)
        y32 = dev_fft(x32)
        ref = dev_fft(x32.astype(np.complex128)).astype(np.complex64)
        worst = max(worst, relerr(y32, ref) / np.finfo(np.float32).eps)
    assert worst <= bound, worst


FAST_LENGTHS = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 3, 9, 27, 81,
                243, 729, 2187, 6561, 1000, 25, 40, 125, 200, 625, 800, 5000]


@pytest.mark.parametrize("n", FAST_LENGTHS)
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_specialised_equals_generic(n, dtype):
    """The length-specialised kernels give the generic kernel's bits."""
    import torch
    rng = np.random.default_rng(n)
    B = 5
    x = torch.from_numpy(crandn(rng, (B, n), dtype)).cuda()
    for planner in (F.plan_fft, F.plan_bfft, F.plan_ifft):
        fast = planner(x.T, 1)
        gen = planner(x.T, 1, _flags=F.FB_FLAG_GENERIC_ONLY)
        a = (fast * x.T).T.cpu().numpy()
        b = (gen * x.T).T.cpu().numpy()
        assert np.array_equal(a, b), (n, planner.__name__, fast.describe(x.T), gen.describe(x.T))
        ref = oracle.fft_nd(x.T.cpu().numpy(), 1, fast.dir, prec="f128") * fast.scale
        assert relerr(a, ref.T) <= tol(dtype, n)


# ----------------------------------------------------------------------- 2D
@pytest.mark.parametrize("N", [8, 11, 15, 16, 27, 100])
def test_delta_2d(N):
    for f in (F.fft, F.bfft):
        y = f(np.ones((N, N), np.complex128))
        ref = np.zeros((N, N))
        ref[0, 0] = N * N
        assert np.allclose(y, ref)


@pytest.mark.parametrize("n", list(range(1, 65, 3)) + [64])
def test_2d_against_oracle(n):
    # test/twodim/complex_forward.jl:15-27, sizes (m, n) with m in n:n+1
    for m in (n, n + 1):
        rng = np.random.default_rng(1000 * m + n)
        for dtype in (np.complex128, np.complex64):
            X = np.asfortranarray(crandn(rng, (m, n), dtype))
            ref = oracle.fft(X, prec="f128")
            assert relerr(F.fft(X), ref) <= tol(dtype, m * n)
            assert relerr(F.ifft(F.fft(X)), X) <= 10 * tol(dtype, m * n)


@pytest.mark.parametrize("n", [1, 2, 3, 6, 11, 16])
def test_2d_regions_bitwise(n):
    # test/twodim/complex_forward.jl:29-43: fft(x, t) == fft(x, r) == mapslices(fft, x; dims=r)
    rng = np.random.default_rng(n)
    x = np.asfortranarray(crandn(rng, (n, n + 1, n + 2)))
    for r in ([1, 2], [1, 3], [2, 3]):
        a = F.fft(x, tuple(r))
        b = F.fft(x, r)
        assert np.array_equal(a, b)
        keep = [d for d in (1, 2, 3) if d not in r][0]
        for i in range(x.shape[keep - 1]):
            sl = [slice(None)] * 3
            sl[keep - 1] = i
            ref = F.fft(np.asfortranarray(x[tuple(sl)]))
            assert np.array_equal(a[tuple(sl)], ref)


@pytest.mark.parametrize("n,dtype", [(1024, np.complex64), (4096, np.complex64),
                                     (1024, np.complex128), (4096, np.complex128)])
def test_long_strided_axis(n, dtype):
    """Long strided lines take a four-step split (tolerance vs the contiguous
    schedule); FB_FLAG_SAME_SCHEDULE_STRIDED restores bitwise equality."""
    import torch
    rng = np.random.default_rng(n)
    X = torch.from_numpy(crandn(rng, (n, 48), dtype)).cuda()  # column axis 1 strided
    cont = F.fft(X.T.contiguous(), 2).T.cpu().numpy()  # rows are contiguous lines
    y = F.fft(X, 1).cpu().numpy()
    ref = oracle.fft_nd(X.cpu().numpy(), 1, -1, prec="f64", nthreads=NTHR)
    assert relerr(y, ref) <= tol(dtype, n)
    assert relerr(cont, ref) <= tol(dtype, n)
    p = F.plan_fft(X, 1, _flags=F.FB_FLAG_SAME_SCHEDULE_STRIDED)
    assert np.array_equal((p * X).cpu().numpy(), cont), p.describe(X)


def test_2d_regions_on_reshaped():
    # test/twodim/complex_forward.jl:3-13 (`≈`)
    N = 11
    x = np.asfortranarray(np.random.default_rng(1).standard_normal((N, N)))
    y = F.fft(x)
    assert np.allclose(y, F.fft(np.asfortranarray(x.reshape(1, N, N, order="F")), [2, 3])[0])
    assert np.allclose(y, F.fft(np.asfortranarray(x.reshape(1, 1, N, N, 1, order="F")),
                                 [3, 4])[0, 0, :, :, 0])


def test_impulse_3x3x3():
    y = np.zeros((3, 3, 3), complex)
    y[1, 1, 1] = 1
    w1 = -0.5 - np.sqrt(3) * 1j / 2
    w2 = np.conj(w1)
    pages = [[[1, w1, w2], [w1, w2, 1], [w2, 1, w1]],
             [[w1, w2, 1], [w2, 1, w1], [1, w1, w2]],
             [[w2, 1, w1], [1, w1, w2], [w1, w2, 1]]]
    ref = np.empty((3, 3, 3), complex)
    for k in range(3):
        ref[:, :, k] = np.array(pages[k])
    assert np.allclose(F.fft(y), ref)


@pytest.mark.parametrize("sz", [(3, 5, 7), (4, 14, 9), (103, 5, 13), (26, 33, 35, 4), (3,) * 5])
def test_nd_ones(sz):
    # test/ndim/minimal_complex.jl:3-8
    x = np.ones(sz, np.complex128)
    ref = np.zeros(sz, complex)
    ref.flat[0] = np.prod(sz)
    assert np.allclose(F.fft(x, tuple(range(1, len(sz) + 1))), ref, atol=1e-8)


# ---------------------------------------------------------- schedule classes
@pytest.mark.parametrize("n", [2 * 101, 73 * 73, 4 * 4099, 2 ** 15, 2 ** 16 * 3, 17 * 19 * 23,
                               3 ** 10, 10007, 30030, 49 * 121])
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_schedule_classes(n, dtype):
    """Four-step, Bluestein in one kernel and in three, big-prime radices."""
    rng = np.random.default_rng(n)
    x = crandn(rng, (3, n), dtype)  # three contiguous transforms (rows)
    xt = np.asfortranarray(x.T)
    y = F.fft(xt, 1)
    ref = oracle.fft_nd(xt, 1, -1, prec="f64", nthreads=NTHR)
    assert relerr(y, ref) <= tol(dtype, n), F.plan_fft(xt, 1).describe(xt)
    yb = F.bfft(xt, 1)
    refb = oracle.fft_nd(xt, 1, 1, prec="f64", nthreads=NTHR)
    assert relerr(yb, refb) <= tol(dtype, n)


@pytest.mark.parametrize("cut", [3, 5, 8, 73, 200])
def test_bluestein_cutoff_kwarg(cut):
    # BLUESTEIN_CUTOFF (src/plan.jl:81) changes the algorithm, not the result
    rng = np.random.default_rng(cut)
    for n in (5, 7, 35, 97, 143):
        x = crandn(rng, n)
        ref = oracle.fft(x, prec="f128")
        assert relerr(F.fft(x, BLUESTEIN_CUTOFF=cut), ref) <= tol(np.complex128, n)


@pytest.mark.parametrize("n,B,dtype", [(4096, 2600, np.complex64), (1000, 5000, np.complex128)])
def test_host_pipeline_matches_device(n, B, dtype):
    """Host arrays above the chunk size go through the three-stream pipeline
    (copy in / transform / copy out); results equal the device path bitwise."""
    import torch
    rng = np.random.default_rng(n)
    x = crandn(rng, (B, n), dtype)
    for planner in (F.plan_fft, F.plan_ifft):
        host = planner(x.T, 1) * x.T
        dev = (planner(x.T, 1) * torch.from_numpy(x).cuda().T).cpu().numpy()
        assert np.array_equal(host, dev)


def test_repeated_calls_reuse_the_checked_plan():
    """A repeated mul_ on tensors laid out like an earlier call's skips the
    argument checks and reuses that call's plan (same bits); any other layout
    or element type still meets every check."""
    import torch
    rng = np.random.default_rng(5)
    x = torch.from_numpy(crandn(rng, (6, 1000), np.complex64)).cuda().T  # 1000 x 6, column-major
    y = torch.empty_like(x)
    p = F.plan_fft(x, 1)
    first = F.mul_(y, p, x).cpu().clone()
    assert len(p._fast) == 1
    for _ in range(3):
        assert torch.equal(F.mul_(y, p, x).cpu(), first)
    ref = oracle.fft_nd(x.cpu().numpy(), 1, -1, prec="f64", nthreads=NTHR)
    assert relerr(first.numpy(), ref) <= tol(np.complex64, 1000)
    short = x[:999]
    with pytest.raises(F.DimensionMismatch):
        F.mul_(torch.empty_like(short), p, short)
    with pytest.raises(F.ArgumentError):
        F.mul_(y.to(torch.complex128), p, x.to(torch.complex128))
    assert len(p._fast) == 1


def test_lazily_conjugated_and_negated_views():
    """torch's conj() and -x of a view are flags, not storage: an input view
    transforms its values, an output view receives them, and neither layout
    enters the repeated-call shortcut."""
    import torch
    rng = np.random.default_rng(9)
    xh = crandn(rng, (4, 1024), np.complex64)
    x = torch.from_numpy(xh).cuda().T
    p = F.plan_fft(x, 1)
    for view, ref_in in ((x.conj(), np.conj(xh)), (torch._neg_view(x), -xh),
                         (torch._neg_view(x.conj()), -np.conj(xh))):
        assert view.is_conj() or view.is_neg()
        for _ in range(2):  # the second call must not take a cached plan of the storage
            y = (p * view).T.cpu().numpy()
            ref = oracle.fft_batched(ref_in.astype(np.complex128), -1, nthreads=NTHR)
            assert relerr(y, ref) <= tol(np.complex64, 1024)
    out = torch.empty_like(x).conj()
    for _ in range(2):
        F.mul_(out, p, x)
        ref = oracle.fft_batched(xh.astype(np.complex128), -1, nthreads=NTHR)
        assert relerr(out.T.resolve_conj().cpu().numpy(), ref) <= tol(np.complex64, 1024)
    torch.cuda.synchronize()


def test_in_place_and_strided():
    import torch
    rng = np.random.default_rng(5)
    x = crandn(rng, (64, 48))
    t = to_dev(x)
    p = F.plan_fft(t, 2)
    ref = oracle.fft(x, 2, prec="f128")
    F.mul_(t, p, t)  # in place
    assert relerr(t.cpu().numpy(), ref) <= tol(np.complex128, 48)
    # a strided view: every other row
    base = to_dev(crandn(rng, (20, 30)))
    view = base[::2]
    y = F.fft(view, 2)
    assert relerr(y.cpu().numpy(), oracle.fft(view.cpu().numpy(), 2, prec="f128")) <= tol(
        np.complex128, 30)
    torch.cuda.synchronize()


# ------------------------------------------------------- the configurations
def test_config1_n1024_c64_round_trip():
    rng = np.random.default_rng(1)
    x = crandn(rng, 1024)
    y = dev_fft(x)
    assert relerr(y, oracle.fft(x, prec="f128")) <= tol(np.complex128, 1024)
    assert relerr(y, oracle.fft(x, prec="f64")) <= tol(np.complex128, 1024)  # FFTA arithmetic
    z = dev_fft(y, None, 1)
    assert relerr(z, 1024 * x) <= tol(np.complex128, 1024)


@pytest.mark.parametrize("N", [4096, 19683, 27648, 2 ** 20])
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_config2_batched(N, dtype):
    B = 2 ** 24 // N
    rng = np.random.default_rng(N)
    x = crandn(rng, (B, N), dtype)  # row b = column b of the Julia N x B matrix
    xt = np.asfortranarray(x.T)
    import torch
    t = torch.from_numpy(x).cuda()
    for direction in (-1, 1):
        p = (F.plan_fft if direction == -1 else F.plan_bfft)(xt, 1)
        # device run on the (N, B) column-major view of the row-major tensor
        y = (p * t.T).T.cpu().numpy()
        ref = oracle.fft_batched(x.astype(np.complex128), direction, nthreads=NTHR)
        e = relerr(y, ref)
        assert e <= tol(dtype, N), (N, direction, e)
        if dtype == np.complex64 and N == 4096:
            assert e <= 1e-6


@pytest.mark.parametrize("N,B,dtype", [(2 ** 15, 8, np.complex64), (2 ** 20, 2, np.complex64),
                                       (27648, 6, np.complex64), (2 ** 14 * 3, 4, np.complex128),
                                       (2 ** 20, 2, np.complex128)])
def test_four_step_specialised_equals_generic(N, B, dtype):
    """Four-step passes on the specialised tile kernels give the generic
    kernel's bits: both take the twiddle on a lean pass's loads as the same
    product of two table entries."""
    import torch
    rng = np.random.default_rng(N + B)
    x = torch.from_numpy(crandn(rng, (B, N), dtype)).cuda()
    for planner in (F.plan_fft, F.plan_bfft):
        fast = planner(x.T, 1)
        gen = planner(x.T, 1, _flags=F.FB_FLAG_GENERIC_ONLY)
        df, dg = fast.describe(x.T), gen.describe(x.T)
        assert "FOUR" in df and "tile" in df and "tile" not in dg, (df, dg)
        a = (fast * x.T).T.cpu().numpy()
        b = (gen * x.T).T.cpu().numpy()
        assert np.array_equal(a, b), (N, planner.__name__, df, dg)
        ref = oracle.fft_batched(x.cpu().numpy().astype(np.complex128), fast.dir, nthreads=NTHR)
        assert relerr(a, ref) <= tol(dtype, N)


CONFIG3 = [(1009, 64), (65537, 16), (1000003, 1), (2 ** 8 * 4099, 4)]


def _blue_run(x, direction):
    import torch
    t = torch.from_numpy(x).cuda()
    planner = F.plan_fft if direction == -1 else F.plan_bfft
    y = (planner(np.asfortranarray(x.T), 1) * t.T).T.cpu().numpy()
    torch.cuda.synchronize()
    return y


@pytest.mark.parametrize("N,B", CONFIG3)
def test_config3_bluestein_tone(N, B):
    """Configuration 3 as stated: i.i.d. complex normal noise (sigma 1 per part)
    plus a unit-amplitude tone at a seeded bin k0.  The tone's peak (N) must
    land at k0 and the whole spectrum -- noise included, which carries almost
    all of the norm here -- must match the FP64 oracle."""
    rng = np.random.default_rng(N)
    x = crandn(rng, (B, N))
    k0 = int(rng.integers(0, N))
    x = (x + np.exp(2j * np.pi * k0 * np.arange(N) / N)).astype(np.complex64)
    y = _blue_run(x, -1)
    ref = oracle.fft_batched(x.astype(np.complex128), -1, nthreads=NTHR)
    assert relerr(y, ref) <= tol(np.complex64, N)
    assert np.all(np.argmax(np.abs(y), axis=1) == k0)


@pytest.mark.parametrize("direction", [-1, 1])
@pytest.mark.parametrize("N,B", CONFIG3)
def test_config3_bluestein_noise(N, B, direction):
    """Noise only, both directions, at the configuration-3 lengths (BLUE1 for
    1009; three-pass Bluestein for 65537 and 1000003, whose pads above 2^18
    take their twiddles from root tables on the passes' stores; a four-step
    split with a Bluestein pass for 2^8 * 4099).  rel-L2 against the FP64
    oracle within 4 eps(Float32) log2 N, and per transform as well, so no
    column can hide behind the others."""
    rng = np.random.default_rng(N + 7 * direction)
    x = crandn(rng, (B, N), np.complex64)
    y = _blue_run(x, direction)
    ref = oracle.fft_batched(x.astype(np.complex128), direction, nthreads=NTHR)
    assert relerr(y, ref) <= tol(np.complex64, N)
    for b in range(B):
        assert relerr(y[b], ref[b]) <= tol(np.complex64, N), b


@pytest.mark.parametrize("m,n", [(4096, 4096), (2187, 2048), (1000, 1000)])
def test_config4_2d(m, n):
    rng = np.random.default_rng(m + n)
    X = crandn(rng, (n, m), np.complex64)  # row-major (n, m) = Julia column-major (m, n)
    import torch
    t = torch.from_numpy(X).cuda()
    y = F.fft(t.T).T.cpu().numpy()
    ref = oracle.fft(np.asfortranarray(X.T.astype(np.complex128)), nthreads=NTHR).T
    assert relerr(y, ref) <= tol(np.complex64, m * n)


@pytest.mark.parametrize("n,B,dtype", [(4096, 8, np.complex64), (2 ** 20, 16, np.complex64),
                                       (27648, 7, np.complex128), (1000003, 3, np.complex64),
                                       (1009, 9, np.complex64), (24576, 5, np.complex64)])
def test_execute_batch_prefix(n, B, dtype):
    """fb_execute_batch runs a batched plan on its first `batch` columns
    (mul! on the leading columns): the same bits as the full plan there,
    nothing written beyond -- across direct, four-step (L2-chunked), and
    Bluestein schedules."""
    import ctypes
    import torch
    from ffta_b200 import _lib
    rng = np.random.default_rng(n + B)
    x = torch.from_numpy(crandn(rng, (B, n), dtype)).cuda()
    h = ctypes.c_void_p()
    dt = _lib.FB_C32 if dtype == np.complex64 else _lib.FB_C64
    assert _lib.lib.fb_plan_create(ctypes.byref(h), n, dt, -1, B, 1, n, 1, n, 73, 0) == 0
    try:
        full = torch.empty_like(x)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert _lib.lib.fb_execute(h, ctypes.c_void_p(x.data_ptr()),
                                   ctypes.c_void_p(full.data_ptr()), st) == 0
        for nb in sorted({1, B // 2 + 1, B}):
            y = torch.full_like(x, float("nan"))
            assert _lib.lib.fb_execute_batch(h, ctypes.c_void_p(x.data_ptr()),
                                             ctypes.c_void_p(y.data_ptr()), nb, st) == 0, \
                _lib.last_error()
            torch.cuda.synchronize()
            assert torch.equal(y[:nb], full[:nb]), nb
            assert torch.isnan(y[nb:]).all(), nb
        bad = _lib.lib.fb_execute_batch(h, ctypes.c_void_p(x.data_ptr()),
                                        ctypes.c_void_p(full.data_ptr()), B + 1, st)
        assert bad == _lib.FB_ERR_DIMENSION_MISMATCH
    finally:
        _lib.lib.fb_plan_destroy(h)
