"""ffta_b200 -- FFTA.jl's complex transform API over the sm_100a C ABI.

Mirrors the plan/transform interface FFTA implements for AbstractFFTs
(FFTA src/plan.jl):

  plan_fft(x, region; BLUESTEIN_CUTOFF=73)   src/plan.jl:71-72, 77-100
  plan_bfft(x, region; ...)                  src/plan.jl:74-75
  p * x                                      src/plan.jl:374-384
  mul_(y, p, x)      (Julia's mul!)          src/plan.jl:157-285
  size(p), size(p, i)                        src/plan.jl:36-47
  fft / bfft / ifft  (AbstractFFTs front-ends: ifft is bfft scaled by 1/n)

Regions are Julia's: 1-based dimension numbers (dim d is numpy/torch axis
d-1), an int, a tuple, a list or a range.  Arrays are numpy arrays (host) or
torch CUDA tensors (device) of complex64/complex128; float32/float64 inputs
are promoted to complex as AbstractFFTs does.  Every other element type raises
ArgumentError: there is no CPU fallback.  Errors raise the Python analogues of
FFTA's exceptions (DimensionMismatch, ArgumentError, DomainError) with FFTA's
messages.
"""
from __future__ import annotations

import ctypes
from collections.abc import Sequence

import numpy as np

from . import _lib
from ._lib import lib

__all__ = [
    "FFT_FORWARD", "FFT_BACKWARD", "DEFAULT_BLUESTEIN_CUTOFF", "DimensionMismatch",
    "ArgumentError", "DomainError", "CudaError", "UnsupportedError", "FFTAPlan_cx", "plan_fft",
    "plan_bfft", "plan_ifft", "fft", "bfft", "ifft", "mul_", "size", "version", "FFTAPlan_re",
    "plan_rfft", "plan_brfft", "plan_irfft", "rfft", "brfft", "irfft", "autotune",
    "save_tuning", "load_tuning",
]

FFT_FORWARD = -1  # src/callgraph.jl:1
FFT_BACKWARD = 1
DEFAULT_BLUESTEIN_CUTOFF = 73  # src/callgraph.jl:44


class DimensionMismatch(Exception):
    """Julia's DimensionMismatch."""


class ArgumentError(Exception):
    """Julia's ArgumentError."""


class DomainError(Exception):
    """Julia's DomainError."""


class CudaError(RuntimeError):
    """A CUDA runtime failure, or no CUDA device (there is no CPU fallback)."""


class UnsupportedError(RuntimeError):
    """A length this build has no kernel schedule for."""


_STATUS = {
    _lib.FB_ERR_DIMENSION_MISMATCH: DimensionMismatch,
    _lib.FB_ERR_ARGUMENT: ArgumentError,
    _lib.FB_ERR_DOMAIN: DomainError,
    _lib.FB_ERR_CUDA: CudaError,
    _lib.FB_ERR_UNSUPPORTED: UnsupportedError,
    _lib.FB_ERR_OUT_OF_MEMORY: MemoryError,
}


def _check(rc: int) -> None:
    if rc != _lib.FB_OK:
        raise _STATUS.get(rc, RuntimeError)(_lib.last_error())


def version() -> str:
    return lib.fb_version().decode()


# ------------------------------------------------------------------ arrays
def _is_torch(x) -> bool:
    t = type(x)
    return t.__module__.startswith("torch") and t.__name__ == "Tensor"


def _torch():
    import torch
    return torch


def _complex_dtype_name(x) -> str:
    """'c64' / 'c128' after AbstractFFTs' real -> complex promotion, else raise."""
    if _is_torch(x):
        torch = _torch()
        m = {torch.complex64: "c64", torch.complex128: "c128", torch.float32: "f32",
             torch.float64: "f64"}
        k = m.get(x.dtype)
    else:
        k = {np.dtype(np.complex64): "c64", np.dtype(np.complex128): "c128",
             np.dtype(np.float32): "f32", np.dtype(np.float64): "f64"}.get(np.asarray(x).dtype)
    if k is None:
        raise ArgumentError(
            f"element type {x.dtype} is not supported: only ComplexF32/ComplexF64 (and "
            "Float32/Float64, promoted to complex) run on the GPU, and there is no CPU fallback")
    return {"f32": "c64", "f64": "c128"}.get(k, k)


def _promote(x):
    """Apply AbstractFFTs' complexfloat promotion; reject other element types."""
    kind = _complex_dtype_name(x)
    if _is_torch(x):
        torch = _torch()
        # torch keeps conj() and negation of a view as flags on the tensor,
        # not in its storage; the kernels read the storage, so materialise them
        x = x.resolve_conj().resolve_neg()
        want = torch.complex64 if kind == "c64" else torch.complex128
        return x if x.dtype == want else x.to(want)
    x = np.asarray(x)
    want = np.complex64 if kind == "c64" else np.complex128
    return x if x.dtype == want else x.astype(want)


def _shape(x):
    return tuple(int(s) for s in x.shape)


def _elem_strides(x):
    """Element strides of x, or None when x needs a copy (negative/odd strides)."""
    if _is_torch(x):
        if x.is_conj() or x.is_neg():
            return None  # lazily conjugated/negated view: the storage is not the values
        st = tuple(int(s) for s in x.stride())
        return None if any(s < 0 for s in st) else st
    item = x.itemsize
    st = []
    for s in x.strides:
        if s < 0 or s % item:
            return None
        st.append(s // item)
    return tuple(st)


def _similar(x):
    """Julia's similar(x): a new array of the same shape and element type."""
    if _is_torch(x):
        torch = _torch()
        if x.is_conj() or x.is_neg():
            return torch.empty(x.shape, dtype=x.dtype, device=x.device)
        if x.is_contiguous():
            return torch.empty_like(x, memory_format=torch.contiguous_format)
        # keep a dense layout with the same dim order when x is dense
        return torch.empty_like(x)
    order = "F" if (x.flags.f_contiguous and not x.flags.c_contiguous) else "C"
    return np.empty(x.shape, dtype=x.dtype, order=order)


def _normalize_region(region, nd):
    """Return (stored region object, sorted tuple) following FFTA's _sort."""
    if region is None:
        region = range(1, nd + 1)
    if isinstance(region, (int, np.integer)):
        r = int(region)
        return r, (r,)
    if isinstance(region, range):
        vals = tuple(region)
        return region if vals == tuple(sorted(vals)) else sorted(vals), tuple(sorted(vals))
    if isinstance(region, tuple):
        vals = tuple(int(v) for v in region)
        return tuple(sorted(vals)), tuple(sorted(vals))
    if isinstance(region, Sequence) or isinstance(region, np.ndarray):
        vals = [int(v) for v in region]
        return sorted(vals), tuple(sorted(vals))
    raise ArgumentError(f"invalid region {region!r}")


def _region_isvalid_nd(r, N):
    """region_isvalid(r, N), src/plan.jl:350-359 (ND plan, ND array)."""
    if isinstance(r, int):
        return r == N == 1
    return list(r) == list(range(1, N + 1))


def _region_isvalid_md(r, M):
    """region_isvalid(r, M, N), src/plan.jl:350-370 (M-dim plan, N-dim array)."""
    if isinstance(r, int):
        return M == 1
    vals = list(r)
    if len(vals) != M:
        return False
    return all(a < b for a, b in zip(vals, vals[1:]))


# ------------------------------------------------------------------ plans
class FFTAPlan_cx:
    """A complex transform plan (FFTA's FFTAPlan_cx, src/plan.jl:9-20).

    Holds the transform sizes and the region; the device schedules (one C plan
    per array layout it is applied to) are created on first use and cached.
    """

    def __init__(self, sizes, region, direction, dtype_kind, cutoff, scale=1.0, flags=0):
        self._flags = int(flags)
        self._sizes = tuple(sizes)
        self.region = region
        self.dir = direction
        self._kind = dtype_kind  # "c64" / "c128"
        self.BLUESTEIN_CUTOFF = cutoff
        self.scale = scale
        self._cplans = {}
        # layouts of (x, y) device tensors that passed every check of mul_
        # without a copy -> their C plan (owned by _cplans)
        self._fast = {}

    # -- AbstractFFTs surface
    def size(self, i=None):
        """Base.size(p) / Base.size(p, i) (src/plan.jl:36-47)."""
        if i is None:
            return self._sizes
        i = int(i)
        if i < 1:
            raise DomainError(f"{i}: No non-positive dimensions")
        if i > len(self._sizes):
            return 1
        return self._sizes[i - 1]

    @property
    def ndims(self):
        return len(self._sizes)

    def __mul__(self, x):
        """p * x (src/plan.jl:374-384): allocate y = similar(x) and mul!."""
        x = self._accept(x)
        y = _similar(x)
        return mul_(y, self, x)

    def __matmul__(self, x):
        return self.__mul__(x)

    def __del__(self):
        try:
            for h in self._cplans.values():
                lib.fb_plan_destroy(h)
        except Exception:
            pass

    def describe(self, x) -> str:
        """The device schedule used for arrays shaped and strided like x."""
        x = self._accept(x)
        h = self._cplan(x, x)
        buf = ctypes.create_string_buffer(4096)
        _check(lib.fb_plan_describe(h, buf, len(buf)))
        return buf.value.decode()

    def device_bytes(self, x) -> int:
        x = self._accept(x)
        h = self._cplan(x, x)
        v = ctypes.c_size_t()
        _check(lib.fb_plan_device_bytes(h, ctypes.byref(v)))
        return int(v.value)

    # -- internals
    def _accept(self, x):
        if not _is_torch(x):
            x = np.asarray(x)
        kind = _complex_dtype_name(x)
        if kind != self._kind:
            raise ArgumentError(
                f"plan is for {self._kind} arrays but got {kind} (FFTA plans are typed, "
                "src/plan.jl:9)")
        return _promote(x)

    def _regions_for(self, nd):
        r = self.region
        if nd == 1 and self.ndims == 1:
            return [1]  # a 1D plan applied to a vector (src/plan.jl:157-167)
        return [r] if isinstance(r, int) else list(r)

    def _cplan(self, y, x):
        xs, ys = _elem_strides(x), _elem_strides(y)
        key = (_shape(x), xs, ys)
        h = self._cplans.get(key)
        if h is not None:
            return h
        nd = x.ndim
        dims = (ctypes.c_int64 * nd)(*_shape(x))
        ist = (ctypes.c_int64 * nd)(*xs)
        ost = (ctypes.c_int64 * nd)(*ys)
        reg = self._regions_for(nd)
        creg = (ctypes.c_int32 * max(1, len(reg)))(*reg)
        handle = ctypes.c_void_p()
        dt = _lib.FB_C32 if self._kind == "c64" else _lib.FB_C64
        _check(lib.fb_plan_create_nd(ctypes.byref(handle), dt, self.dir, nd, dims, ist, ost,
                                     len(reg), creg, int(self.BLUESTEIN_CUTOFF), self._flags))
        if self.scale != 1.0:
            _check(lib.fb_plan_set_scale(handle, float(self.scale)))
        self._cplans[key] = handle
        return handle


def _make_plan(x, region, direction, cutoff, scale_inverse=False, flags=0):
    if not _is_torch(x):
        x = np.asarray(x)
    kind = _complex_dtype_name(x)
    nd = x.ndim
    stored, srt = _normalize_region(region, nd)
    shape = _shape(x)
    sizes = []
    for r in srt:
        if r < 1 or r > nd:
            # FFTA reads size(x, R) which is 1 beyond ndims; CallGraph(1) is fine,
            # and mul! later rejects the region.
            sizes.append(1 if r > nd else 0)
        else:
            sizes.append(shape[r - 1])
    for s in sizes:
        if s <= 0:
            raise DimensionMismatch("Array length must be strictly positive")
    scale = 1.0
    if scale_inverse:
        scale = 1.0 / float(np.prod(sizes))
    return FFTAPlan_cx(sizes, stored, direction, kind, int(cutoff), scale, flags)


FB_FLAG_GENERIC_ONLY = 1  # include/fftab200.h: generic kernels only (for tests)
FB_FLAG_SAME_SCHEDULE_STRIDED = 2  # strided axes bit-identical to contiguous ones
FB_FLAG_STREAM = 4  # persistent bulk-copy kernel for contiguous lines (bit-identical)
FB_FLAG_TENSOR_STAGE = 8  # C32: first radix-16 stage on the tensor cores (split BF16)
FB_FLAG_TMA = 16  # strided passes load tiles by tensor copies (opt-in; bit-identical)
FB_FLAG_TUNE_RADIX = 32  # autotune also chooses the radix program (results not bitwise equal)
FB_SERVER_NO_GRAPHS = 1  # fb_server_create: no CUDA-graph replay of recurring multi-pass requests
FB_SERVER_NO_PERSISTENT = 2  # fb_server_create: no resident kernel; small requests in descriptor launches
FB_SERVER_SERIAL = 4  # fb_server_create: one request at a time, one plan launch each (the plain path)


def plan_fft(x, region=None, *, BLUESTEIN_CUTOFF=DEFAULT_BLUESTEIN_CUTOFF, _flags=0, **_kwargs):
    """AbstractFFTs.plan_fft (FFTA src/plan.jl:71-72)."""
    return _make_plan(x, region, FFT_FORWARD, BLUESTEIN_CUTOFF, flags=_flags)


def plan_bfft(x, region=None, *, BLUESTEIN_CUTOFF=DEFAULT_BLUESTEIN_CUTOFF, _flags=0, **_kwargs):
    """AbstractFFTs.plan_bfft (FFTA src/plan.jl:74-75): unnormalised inverse."""
    return _make_plan(x, region, FFT_BACKWARD, BLUESTEIN_CUTOFF, flags=_flags)


def plan_ifft(x, region=None, *, BLUESTEIN_CUTOFF=DEFAULT_BLUESTEIN_CUTOFF, _flags=0, **_kwargs):
    """AbstractFFTs.plan_ifft: plan_bfft scaled by 1/prod(sizes), fused in-kernel."""
    return _make_plan(x, region, FFT_BACKWARD, BLUESTEIN_CUTOFF, scale_inverse=True,
                      flags=_flags)


def size(p: FFTAPlan_cx, i=None):
    return p.size(i)


def _fast_key(y, x):
    """Layout key of two complex CUDA tensors (shapes, strides, type,
    devices), or None for anything else."""
    if not (_is_torch(x) and _is_torch(y)):
        return None
    dt = x.dtype
    if dt is not y.dtype or not dt.is_complex or not x.is_cuda or not y.is_cuda:
        return None
    if x.is_conj() or x.is_neg() or y.is_conj() or y.is_neg():
        return None
    return (x.shape, x.stride(), y.shape, y.stride(), dt, x.device.index, y.device.index)


def _execute_device(h, x, y):
    """fb_execute on the current stream of x's device."""
    torch = _torch()
    dev = x.device
    stream = torch.cuda.current_stream(dev).cuda_stream
    args = (h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(stream))
    if dev.index == torch.cuda.current_device():
        _check(lib.fb_execute(*args))
    else:
        with torch.cuda.device(dev):
            _check(lib.fb_execute(*args))


def mul_(y, p: FFTAPlan_cx, x):
    """LinearAlgebra.mul!(y, p, x) with FFTA's argument checks (src/plan.jl:157-285).

    Device tensors laid out like an earlier call's that passed those checks
    without a copy (same shapes, strides, type and devices) go straight to
    the plan that call used: the checks depend on nothing else."""
    fk = _fast_key(y, x)
    if fk is not None:
        h = p._fast.get(fk)
        if h is not None:
            _execute_device(h, x, y)
            return y
    x_arg = x
    x = p._accept(x)
    if _is_torch(y) != _is_torch(x):
        raise ArgumentError("input and output must both be host arrays or both device tensors")
    if not _is_torch(y):
        y = np.asarray(y)
    if _complex_dtype_name(y) != p._kind or (not _is_torch(y) and y.dtype != x.dtype):
        raise ArgumentError("output element type must match the plan")
    N, M = x.ndim, p.ndims
    r = p.region
    xs, ys = _shape(x), _shape(y)
    if M == 1:
        # 1D plan: vector (src/plan.jl:157-167) or N-D array (src/plan.jl:170-192)
        if xs != ys:
            raise DimensionMismatch(f"input array has axes {xs}, but output array has axes {ys}")
        R1 = r if isinstance(r, int) else (list(r)[0] if len(list(r)) == 1 else None)
        if R1 is None:
            raise DimensionMismatch("Region is invalid.")
        if N == 1:
            if p.size() != xs:
                raise DimensionMismatch(f"plan has axes {p.size()}, but input array has axes {xs}")
        else:
            if R1 < 1 or R1 > N:
                raise DimensionMismatch("Plan region is outside array dimensions.")
            if p.size(1) != xs[R1 - 1]:
                raise DimensionMismatch(
                    f"plan has size {p.size(1)}, but input array has size {xs[R1 - 1]} along "
                    f"region {R1}")
    elif M == N:
        # ND plan, ND array (src/plan.jl:210-222)
        if xs != ys:
            raise DimensionMismatch(f"input array has axes {xs}, but output array has axes {ys}")
        if p.size() != xs:
            raise DimensionMismatch(f"plan has size {p.size()}, but input array has size {xs}")
        if not _region_isvalid_nd(r, N):
            raise DimensionMismatch("Plan region is outside array dimensions.")
    else:
        # M-dim plan on an N-dim array (src/plan.jl:260-272)
        if xs != ys:
            raise DimensionMismatch(f"input array has axes {xs}, but output array has axes {ys}")
        if not _region_isvalid_md(r, M):
            raise DimensionMismatch("Region is invalid.")
        vals = list(r)
        if M > N or vals[0] < 1 or vals[-1] > N:
            raise DimensionMismatch("Plan region is outside array dimensions.")
        for k, d in enumerate(vals):
            if p.size(k + 1) != xs[d - 1]:
                raise DimensionMismatch(
                    f"plan has size {p.size()}, but input array has size {xs}")
    if x.size == 0:
        return y
    # The C plan needs element strides; copy views it cannot address.
    if _elem_strides(x) is None:
        x = x.contiguous() if _is_torch(x) else np.ascontiguousarray(x)
    y_target = y
    if _elem_strides(y) is None:
        y = _similar(y)
    h = p._cplan(y, x)
    if _is_torch(x):
        if not x.is_cuda or not y.is_cuda:
            raise ArgumentError("torch tensors must live on a CUDA device")
        _execute_device(h, x, y)
        if fk is not None and x is x_arg and y is y_target:
            p._fast[fk] = h
    else:
        _check(lib.fb_execute_host(h, ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(y.ctypes.data),
                                   None))
    if y is not y_target:
        y_target[...] = y
        y = y_target
    return y


def _apply(planner, x, region, **kw):
    x = _promote(x if _is_torch(x) else np.asarray(x))
    p = planner(x, region, **kw)
    return p * x


def fft(x, region=None, **kw):
    """AbstractFFTs fft(x, region) -> plan_fft(x, region) * x."""
    return _apply(plan_fft, x, region, **kw)


def bfft(x, region=None, **kw):
    """AbstractFFTs bfft(x, region) -> plan_bfft(x, region) * x (unnormalised)."""
    return _apply(plan_bfft, x, region, **kw)


def ifft(x, region=None, **kw):
    """AbstractFFTs ifft: bfft scaled by 1/prod(sizes along region)."""
    return _apply(plan_ifft, x, region, **kw)


# -------------------------------------------------------- real transforms
def _real_kind(x) -> str:
    """'f32' / 'f64' for real inputs, 'c64' / 'c128' for complex, else raise."""
    if _is_torch(x):
        torch = _torch()
        k = {torch.float32: "f32", torch.float64: "f64", torch.complex64: "c64",
             torch.complex128: "c128"}.get(x.dtype)
    else:
        k = {np.dtype(np.float32): "f32", np.dtype(np.float64): "f64",
             np.dtype(np.complex64): "c64", np.dtype(np.complex128): "c128"}.get(
                 np.asarray(x).dtype)
    if k is None:
        raise ArgumentError(f"element type {x.dtype} is not supported: only Float32/Float64 "
                            "(and their complex types) run on the GPU, and there is no CPU "
                            "fallback")
    return k


def _col_major(x):
    """x as contiguous column-major memory (Julia layout) plus its dims."""
    if _is_torch(x):
        perm = tuple(range(x.ndim - 1, -1, -1))
        return x.permute(perm).contiguous(), tuple(int(s) for s in x.shape)
    return np.asfortranarray(x), tuple(int(s) for s in x.shape)


class FFTAPlan_re:
    """A real transform plan (FFTA's FFTAPlan_re, src/plan.jl:22-34).

    dir FFT_FORWARD: rfft (real input, n/2+1 outputs along the first region
    dim); FFT_BACKWARD: brfft of length `flen` (complex input, real output).
    """

    def __init__(self, sizes, region, direction, prec, flen, cutoff, scale=1.0):
        self._sizes = tuple(sizes)
        self.region = region
        self.dir = direction
        self._prec = prec  # "f32" / "f64"
        self.flen = int(flen)
        self.BLUESTEIN_CUTOFF = cutoff
        self.scale = scale
        self._cplans = {}

    def size(self, i=None):
        """Base.size (src/plan.jl:36-47): the real length first."""
        sz = (self.flen,) + self._sizes[1:]
        if i is None:
            return sz
        i = int(i)
        if i < 1:
            raise DomainError(f"{i}: No non-positive dimensions")
        return sz[i - 1] if i <= len(sz) else 1

    @property
    def ndims(self):
        return len(self._sizes)

    def __del__(self):
        try:
            for h in self._cplans.values():
                lib.fb_plan_destroy(h)
        except Exception:
            pass

    def _regions(self):
        r = self.region
        return [r] if isinstance(r, int) else list(r)

    def describe(self, dims) -> str:
        """The device schedule for a real array of `dims` (Julia order)."""
        buf = ctypes.create_string_buffer(8192)
        _check(lib.fb_plan_describe(self._handle(tuple(int(d) for d in dims)), buf, len(buf)))
        return buf.value.decode()

    def _handle(self, dims):
        h = self._cplans.get(dims)
        if h is None:
            reg = self._regions()
            cd = (ctypes.c_int64 * len(dims))(*dims)
            cr = (ctypes.c_int32 * len(reg))(*reg)
            hh = ctypes.c_void_p()
            dt = _lib.FB_C32 if self._prec == "f32" else _lib.FB_C64
            _check(lib.fb_plan_create_real(ctypes.byref(hh), dt, self.dir, len(dims), cd,
                                           len(reg), cr, int(self.BLUESTEIN_CUTOFF), 0))
            if self.scale != 1.0:
                _check(lib.fb_plan_set_scale(hh, float(self.scale)))
            self._cplans[dims] = hh
            h = hh
        return h

    def __mul__(self, x):
        kind = _real_kind(x)
        vec = x.ndim == 1
        what = "vectors" if vec else "arrays"
        reg = self._regions()
        if kind in ("f32", "f64"):
            # src/plan.jl:390-393, 508-511, 532-535
            if self.dir != FFT_FORWARD:
                raise ArgumentError(f"only FFT_FORWARD supported for real {what}")
            if kind != self._prec:
                raise ArgumentError("plan is for another precision")
            dims = tuple(int(s) for s in x.shape)
            if reg[-1] > x.ndim or reg[0] < 1:
                raise DimensionMismatch("Plan region is outside array dimensions.")
            got = tuple(dims[r - 1] for r in reg)
            if got != (self.flen,) + self._sizes[1:]:
                raise DimensionMismatch(
                    f"plan has size {self.size()}, but input array has size {got}")
            out_dims = list(dims)
            out_dims[reg[0] - 1] = self.flen // 2 + 1
            return self._run(x, dims, tuple(out_dims), complex_out=True)
        # complex input: brfft (src/plan.jl:457-460, 517-520, 545-548)
        if self.dir != FFT_BACKWARD:
            raise ArgumentError(f"only FFT_BACKWARD supported for complex {what}")
        if {"c64": "f32", "c128": "f64"}[kind] != self._prec:
            raise ArgumentError("plan is for another precision")
        xs = tuple(int(s) for s in x.shape)
        if reg[-1] > x.ndim or reg[0] < 1:
            raise DimensionMismatch("Plan region is outside array dimensions.")
        rlen = self.flen // 2 + 1
        if xs[reg[0] - 1] != rlen:
            raise DimensionMismatch(
                f"real {len(reg)}D plan has size {self.flen}. Dimension of input array along "
                f"region {reg[0]} should have size {rlen}, but has size {xs[reg[0] - 1]}")
        if tuple(xs[r - 1] for r in reg[1:]) != self._sizes[1:]:
            raise DimensionMismatch(f"real {len(reg)}D plan has size {self.size()}")
        dims = list(xs)
        dims[reg[0] - 1] = self.flen
        return self._run(x, tuple(dims), tuple(dims), complex_out=False)

    def _run(self, x, dims, out_dims, complex_out):
        """Execute on `x`; `dims` are the real-array dims the plan is made for."""
        if any(d == 0 for d in dims):
            raise DimensionMismatch("Array length must be strictly positive")
        h = self._handle(dims)
        xc, _ = _col_major(x)
        if _is_torch(x):
            torch = _torch()
            if complex_out:
                odt = torch.complex64 if self._prec == "f32" else torch.complex128
            else:
                odt = torch.float32 if self._prec == "f32" else torch.float64
            y = torch.empty(tuple(reversed(out_dims)), dtype=odt, device=x.device)
            stream = torch.cuda.current_stream(x.device).cuda_stream
            with torch.cuda.device(x.device):
                _check(lib.fb_execute(h, ctypes.c_void_p(xc.data_ptr()),
                                      ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(stream)))
            return y.permute(tuple(range(y.ndim - 1, -1, -1)))
        if complex_out:
            odt = np.complex64 if self._prec == "f32" else np.complex128
        else:
            odt = np.float32 if self._prec == "f32" else np.float64
        y = np.empty(out_dims, dtype=odt, order="F")
        _check(lib.fb_execute_host(h, ctypes.c_void_p(xc.ctypes.data),
                                   ctypes.c_void_p(y.ctypes.data), None))
        return y


def _real_region(x, region):
    stored, srt = _normalize_region(region, x.ndim)
    if len(srt) > 2:
        raise ArgumentError("only supports 1D and 2D FFTs")
    return stored, srt


def plan_rfft(x, region=None, *, BLUESTEIN_CUTOFF=DEFAULT_BLUESTEIN_CUTOFF, **_kwargs):
    """AbstractFFTs.plan_rfft (FFTA src/plan.jl:102-125)."""
    if not _is_torch(x):
        x = np.asarray(x)
    kind = _real_kind(x)
    if kind not in ("f32", "f64"):
        raise ArgumentError("plan_rfft needs a real array")
    stored, srt = _real_region(x, region)
    shape = tuple(int(s) for s in x.shape)
    sizes = tuple(shape[r - 1] if 1 <= r <= x.ndim else 1 for r in srt)
    if any(v <= 0 for v in sizes):
        raise DimensionMismatch("Array length must be strictly positive")
    return FFTAPlan_re(sizes, stored, FFT_FORWARD, kind, sizes[0], int(BLUESTEIN_CUTOFF))


def plan_brfft(x, len_, region=None, *, BLUESTEIN_CUTOFF=DEFAULT_BLUESTEIN_CUTOFF, _scale=False,
               **_kwargs):
    """AbstractFFTs.plan_brfft(x, len, region) (FFTA src/plan.jl:127-150)."""
    if not _is_torch(x):
        x = np.asarray(x)
    kind = _real_kind(x)
    prec = {"c64": "f32", "c128": "f64", "f32": "f32", "f64": "f64"}[kind]
    stored, srt = _real_region(x, region)
    shape = tuple(int(s) for s in x.shape)
    sizes = (int(len_),) + tuple(shape[r - 1] if 1 <= r <= x.ndim else 1 for r in srt[1:])
    if any(v <= 0 for v in sizes):
        raise DimensionMismatch("Array length must be strictly positive")
    scale = 1.0 / float(np.prod(sizes)) if _scale else 1.0
    return FFTAPlan_re(sizes, stored, FFT_BACKWARD, prec, int(len_), int(BLUESTEIN_CUTOFF), scale)


def plan_irfft(x, len_, region=None, **kw):
    """AbstractFFTs.plan_irfft: plan_brfft scaled by 1/prod(sizes)."""
    return plan_brfft(x, len_, region, _scale=True, **kw)


def rfft(x, region=None, **kw):
    if not _is_torch(x):
        x = np.asarray(x)
    return plan_rfft(x, region, **kw) * x


def brfft(x, len_, region=None, **kw):
    if not _is_torch(x):
        x = np.asarray(x)
    return plan_brfft(x, len_, region, **kw) * x


def irfft(x, len_, region=None, **kw):
    if not _is_torch(x):
        x = np.asarray(x)
    return plan_irfft(x, len_, region, **kw) * x


# ------------------------------------------------------------- autotuner
def autotune(p: FFTAPlan_cx, x, y=None, iters: int = 5):
    """Tune the launch shapes `p` uses for arrays laid out like `x` (device
    tensors; `y` defaults to a scratch output, and both are overwritten).
    Later plans for the same length, type, batch and layout start from the
    result (fb_plan_autotune).  Returns the tuned schedule's description."""
    import torch
    x = p._accept(x)
    if not _is_torch(x):
        raise ArgumentError("autotune needs device tensors")
    if y is None:
        y = _similar(x)
    h = p._cplan(y, x)
    stream = torch.cuda.current_stream(x.device).cuda_stream
    _check(lib.fb_plan_autotune(h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                ctypes.c_void_p(stream), int(iters)))
    return p.describe(x)


def save_tuning(path: str) -> None:
    """Write the process's tuning cache to a text file."""
    _check(lib.fb_tune_cache_save(path.encode()))


def load_tuning(path: str) -> None:
    """Merge a tuning cache file into the process's cache."""
    _check(lib.fb_tune_cache_load(path.encode()))
