"""ctypes front-end of the CPU oracle (``liboracle.so``, built from ffta_oracle.cpp).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module, and only to check or to
time the CPU restatement of FFTA.jl; the product (``ffta.jl_b200``) never does.

The functions take Julia's conventions: arrays are transformed along 1-based
dims (``region``), ``dir`` is -1 for FFT_FORWARD and +1 for FFT_BACKWARD
(FFTA ``src/callgraph.jl:1``), and the Bluestein cutoff defaults to 73
(``src/callgraph.jl:44``).  Precision ``"f32"``/``"f64"`` runs FFTA's own
arithmetic in that precision; ``"f128"`` runs the same algorithm in
``__float128`` and is the high-precision oracle.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

FORWARD = -1
BACKWARD = 1
DEFAULT_BLUESTEIN_CUTOFF = 73
NODE_TYPES = ("COMPOSITE_FFT", "DFT", "POW3_FFT", "POW2RADIX4_FFT", "BLUESTEIN")


class OracleDimensionMismatch(Exception):
    pass


def build() -> str:
    """Compile liboracle.so with the committed Makefile (no-op when current)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        i64p = ctypes.POINTER(ctypes.c_int64)
        L.oracle_fft.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                 i64p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                 ctypes.c_int64, ctypes.c_int]
        L.oracle_fft.restype = ctypes.c_int
        for nm in ("oracle_fft_batched_f32", "oracle_fft_batched_f64"):
            f = getattr(L, nm)
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                          ctypes.c_int, ctypes.c_int64, ctypes.c_int]
            f.restype = ctypes.c_int
        L.oracle_callgraph.argtypes = [ctypes.c_int64, ctypes.c_int64, i64p, ctypes.c_int64]
        L.oracle_callgraph.restype = ctypes.c_int64
        L.oracle_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _check(rc: int):
    if rc == 0:
        return
    msg = lib().oracle_last_error().decode()
    if rc == 1:
        raise OracleDimensionMismatch(msg)
    raise ValueError(msg)


def fft_nd(x, region=None, dir: int = FORWARD, prec: str = "f64",
           cutoff: int = DEFAULT_BLUESTEIN_CUTOFF, nthreads: int = 1) -> np.ndarray:
    """Transform ``x`` along the 1-based dims in ``region`` (default: all).

    Follows FFTA's mul! drivers (src/plan.jl:170-207 and :210-257): dims are
    processed in ascending order, each line gathered, transformed by fft! and
    scattered back.  Returns complex128 (exact widening of the f32 result for
    prec="f32").
    """
    x = np.asarray(x)
    if x.ndim == 0:
        x = x.reshape(1)
    if region is None:
        region = list(range(1, x.ndim + 1))
    elif isinstance(region, (int, np.integer)):
        region = [int(region)]
    region = sorted(int(r) for r in region)
    pidx = {"f32": 0, "f64": 1, "f128": 2}[prec]
    xin = np.asfortranarray(x.astype(np.complex128))
    out = np.empty_like(xin, order="F")
    dims = (ctypes.c_int64 * x.ndim)(*x.shape)
    reg = (ctypes.c_int * len(region))(*[r - 1 for r in region])
    rc = lib().oracle_fft(pidx, xin.ctypes.data, out.ctypes.data, x.ndim, dims, len(region), reg,
                          int(dir), int(cutoff), int(nthreads))
    _check(rc)
    return out


def fft(x, region=None, prec="f64", **kw):
    return fft_nd(x, region, FORWARD, prec, **kw)


def bfft(x, region=None, prec="f64", **kw):
    return fft_nd(x, region, BACKWARD, prec, **kw)


def fft_batched(x: np.ndarray, dir: int = FORWARD, cutoff: int = DEFAULT_BLUESTEIN_CUTOFF,
                nthreads: int = 1) -> np.ndarray:
    """Contiguous batched 1D transforms in the array's own precision.

    ``x`` is (batch, n) C-contiguous complex64/complex128, i.e. a Julia N x batch
    column-major matrix; each row is one column transform (src/plan.jl:194-207).
    Used as the timed CPU baseline: lines are split over ``nthreads`` threads.
    """
    x = np.ascontiguousarray(x)
    batch, n = x.shape
    out = np.empty_like(x)
    if x.dtype == np.complex64:
        rc = lib().oracle_fft_batched_f32(x.ctypes.data, out.ctypes.data, n, batch, int(dir),
                                          int(cutoff), int(nthreads))
    elif x.dtype == np.complex128:
        rc = lib().oracle_fft_batched_f64(x.ctypes.data, out.ctypes.data, n, batch, int(dir),
                                          int(cutoff), int(nthreads))
    else:
        raise TypeError("complex64 or complex128 expected")
    _check(rc)
    return out


def callgraph(n: int, cutoff: int = DEFAULT_BLUESTEIN_CUTOFF):
    """FFTA's CallGraph{T}(n, cutoff).nodes (src/callgraph.jl:133-138) as dicts."""
    cap = 4096
    rows = (ctypes.c_int64 * (6 * cap))()
    cnt = lib().oracle_callgraph(int(n), int(cutoff), rows, cap)
    if cnt < 0:
        raise OracleDimensionMismatch(lib().oracle_last_error().decode())
    out = []
    for i in range(cnt):
        l, r, t, sz, si, so = rows[6 * i:6 * i + 6]
        out.append(dict(left=l, right=r, type=NODE_TYPES[t], sz=sz, s_in=si, s_out=so))
    return out
