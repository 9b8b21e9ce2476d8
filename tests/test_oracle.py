"""Pin the CPU oracle (oracle/ffta_oracle.cpp) before trusting it.

FFTA.jl cannot run here (no Julia), so the oracle is pinned against every
known answer the reference's own tests hold for this path, and against the
50-digit golden DFTs in tests/golden (made by tests/golden/make_golden.py):

  * delta answers: fft(ones(N)) = N e_0, test/onedim/complex_forward.jl:3-11,
    bfft: test/onedim/complex_backward.jl:4-11, 2-D: test/twodim/complex_*.jl
  * the O(N^2) naive DFT for n in 1:64 and 73^2,
    test/onedim/complex_forward.jl:14-24 (fixture test/runtests.jl:12-42)
  * round trip ifft(fft(x)) ~ x, test/onedim/complex_backward.jl:13-20
  * batched == per-slice, exactly, test/onedim/complex_forward.jl:26-32
  * the Float32 twiddle-accuracy bounds of issue #118,
    test/onedim/accuracy.jl:15-57
  * the 3x3x3 impulse table, test/ndim/minimal_complex.jl:9-26
  * the call-graph shapes, src/callgraph.jl:76-126
"""
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "dft_golden.npz"))


def naive_dft(x, sign):
    n = len(x)
    k = np.arange(n)
    e = np.exp(sign * 2j * np.pi * ((np.outer(k, k)) % n) / n)
    return e @ x


def relerr(a, b):
    b = np.asarray(b)
    d = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - b) / (d if d else 1.0)


@pytest.mark.parametrize("N", [8, 11, 15, 16, 27, 100, 275])
def test_delta_forward(N):
    y = oracle.fft(np.ones(N, complex))
    ref = np.zeros(N, complex)
    ref[0] = N
    assert np.abs(y - ref).max() <= 1e-12


@pytest.mark.parametrize("N", [8, 11, 15, 16, 27, 100, 103])
def test_delta_backward(N):
    y = oracle.bfft(np.ones(N, complex))
    ref = np.zeros(N, complex)
    ref[0] = N
    assert np.abs(y - ref).max() <= 1e-12


@pytest.mark.parametrize("N", [8, 11, 15, 16, 27, 100])
def test_delta_2d(N):
    for f in (oracle.fft, oracle.bfft):
        y = f(np.ones((N, N), complex))
        ref = np.zeros((N, N), complex)
        ref[0, 0] = N * N
        assert np.allclose(y, ref, atol=1e-9)


@pytest.mark.parametrize("n", list(range(1, 65)) + [73 * 73])
def test_naive_dft(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    # Julia's `≈` on arrays: norm(a-b) <= sqrt(eps) * max(norm(a), norm(b))
    assert relerr(oracle.fft(x), naive_dft(x, -1)) <= np.sqrt(np.finfo(float).eps)
    assert relerr(oracle.bfft(x), naive_dft(x, +1)) <= np.sqrt(np.finfo(float).eps)


@pytest.mark.parametrize("n", [1, 2, 5, 7, 16, 30, 64])
def test_round_trip(n):
    rng = np.random.default_rng(100 + n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert relerr(oracle.bfft(oracle.fft(x)) / n, x) <= np.sqrt(np.finfo(float).eps)


@pytest.mark.parametrize("n", [1, 4, 7, 12])
def test_batched_equals_per_slice(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n + 1, n + 2)) + 1j * rng.standard_normal((n, n + 1, n + 2))
    for r in (1, 2, 3):
        y = oracle.fft(x, r)
        ax = r - 1
        ref = np.apply_along_axis(lambda v: oracle.fft(v), ax, x)
        assert np.array_equal(y, ref)


@pytest.mark.parametrize("n", [int(s) for s in GOLD["sizes"]])
def test_golden_f64_and_f128(n):
    x = GOLD[f"x_{n}"]
    for f, key in ((oracle.fft, "fwd"), (oracle.bfft, "bwd")):
        ref = GOLD[f"{key}_{n}"]
        e64 = relerr(f(x), ref)
        assert e64 <= 4 * np.finfo(float).eps * max(1.0, np.log2(n)) * 8, (n, key, e64)
        e128 = relerr(f(x, prec="f128"), ref)
        assert e128 <= 2 * np.finfo(float).eps, (n, key, e128)


# (N, bound) from test/onedim/accuracy.jl:15-43
POWERS_OF_2 = [(1 << 4, 3.0), (1 << 5, 3.0), (1 << 6, 3.0), (1 << 7, 3.0), (1 << 8, 4.0),
               (1 << 9, 4.0), (1 << 10, 8.0), (1 << 11, 8.0), (1 << 12, 10.0), (1 << 13, 12.0),
               (1 << 14, 14.0), (1 << 15, 20.0), (1 << 16, 22.0)]
POWERS_OF_3 = [(3, 3.0), (9, 3.0), (27, 3.0), (81, 4.0), (243, 5.0), (729, 7.0), (2187, 10.0),
               (6561, 13.0), (19683, 18.0)]


def worst_eps_ratio(fft32, N, fft64=None):
    """test/onedim/accuracy.jl:45-57 with numpy seeds 1..5 for Julia's Xoshiro."""
    worst = 0.0
    for seed in range(1, 6):
        rng = np.random.default_rng(seed)
        x32 = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
        y32 = fft32(x32)
        ref = (fft64 or oracle.fft)(x32.astype(np.complex128)).astype(np.complex64)
        r = np.linalg.norm(y32.astype(np.complex128) - ref) / np.linalg.norm(ref)
        worst = max(worst, r / np.finfo(np.float32).eps)
    return worst


@pytest.mark.parametrize("N,bound", POWERS_OF_2 + POWERS_OF_3)
def test_oracle_f32_accuracy_bounds(N, bound):
    assert worst_eps_ratio(lambda v: oracle.fft(v, prec="f32"), N) <= bound


def test_impulse_3x3x3():
    y = np.zeros((3, 3, 3), complex)
    y[1, 1, 1] = 1
    w1 = -0.5 - np.sqrt(3) * 1j / 2
    w2 = np.conj(w1)
    # the table of test/ndim/minimal_complex.jl:14-25 (Julia column-major pages)
    pages = [
        [[1, w1, w2], [w1, w2, 1], [w2, 1, w1]],
        [[w1, w2, 1], [w2, 1, w1], [1, w1, w2]],
        [[w2, 1, w1], [1, w1, w2], [w1, w2, 1]],
    ]
    ref = np.empty((3, 3, 3), complex)
    for k in range(3):
        ref[:, :, k] = np.array(pages[k])
    assert np.allclose(oracle.fft(y), ref)


@pytest.mark.parametrize("sz", [(3, 5, 7), (4, 14, 9), (103, 5, 13), (26, 33, 35, 4), (3,) * 5])
def test_nd_ones(sz):
    x = np.ones(sz, complex)
    ref = np.zeros(sz, complex)
    ref.flat[0] = np.prod(sz)
    assert np.allclose(oracle.fft(x), ref, atol=1e-8)


def test_callgraph_shapes():
    g = oracle.callgraph(27648)
    assert [(d["type"], d["sz"], d["s_in"], d["s_out"]) for d in g] == [
        ("COMPOSITE_FFT", 27648, 1, 1), ("POW2RADIX4_FFT", 1024, 27, 27), ("POW3_FFT", 27, 1024, 1)]
    assert [d["type"] for d in oracle.callgraph(1000003)] == ["BLUESTEIN"]
    assert [d["type"] for d in oracle.callgraph(19683)] == ["POW3_FFT"]
    g = oracle.callgraph(2 ** 8 * 4099)
    assert [(d["type"], d["sz"]) for d in g] == [
        ("COMPOSITE_FFT", 1049344), ("POW2RADIX4_FFT", 256), ("BLUESTEIN", 4099)]
    # 275 = 5*5*11 takes the N_cp[idx+1] branch: N1 = 25 (src/callgraph.jl:114-116)
    g = oracle.callgraph(275)
    assert g[0]["type"] == "COMPOSITE_FFT" and g[1]["sz"] == 25
    assert [d["type"] for d in oracle.callgraph(71)] == ["DFT"]
    assert [d["type"] for d in oracle.callgraph(73)] == ["BLUESTEIN"]
    assert [d["type"] for d in oracle.callgraph(73, cutoff=100)] == ["DFT"]


def test_empty_raises_dimension_mismatch():
    with pytest.raises(oracle.OracleDimensionMismatch):
        oracle.fft(np.zeros(0, complex))
