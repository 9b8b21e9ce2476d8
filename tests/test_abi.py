"""The C ABI library loads and exports every symbol include/fftab200.h declares.

No compute calls are made here: without a GPU the library must refuse to plan
(FB_ERR_CUDA, "no CPU fallback") rather than compute anything on the host.
"""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fftab200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_api():
    names = declared_functions()
    for n in ("fb_plan_create", "fb_plan_create_2d", "fb_plan_create_nd", "fb_execute",
              "fb_execute_host", "fb_plan_destroy", "fb_last_error", "fb_plan_size"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from ffta_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers the header exactly
    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_version():
    import ffta_b200
    assert "sm_100a" in ffta_b200.version()


def _no_gpu():
    import torch
    return not torch.cuda.is_available()


@pytest.mark.skipif(not _no_gpu(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback():
    from ffta_b200 import _lib
    h = ctypes.c_void_p()
    rc = _lib.lib.fb_plan_create(ctypes.byref(h), 16, 0, -1, 1, 1, 16, 1, 16, 73, 0)
    assert rc == _lib.FB_ERR_CUDA
    assert "no CPU fallback" in _lib.last_error()


def test_status_codes_before_device():
    """Argument errors are reported before any device work (FFTA's DimensionMismatch)."""
    from ffta_b200 import _lib
    h = ctypes.c_void_p()
    assert _lib.lib.fb_plan_create(ctypes.byref(h), 0, 0, -1, 1, 1, 1, 1, 1, 73, 0) == \
        _lib.FB_ERR_DIMENSION_MISMATCH
    assert "strictly positive" in _lib.last_error()
    assert _lib.lib.fb_plan_create(ctypes.byref(h), 8, 7, -1, 1, 1, 8, 1, 8, 73, 0) == \
        _lib.FB_ERR_ARGUMENT
    dims = (ctypes.c_int64 * 2)(3, 3)
    st = (ctypes.c_int64 * 2)(1, 3)
    reg = (ctypes.c_int32 * 1)(3)
    assert _lib.lib.fb_plan_create_nd(ctypes.byref(h), 0, -1, 2, dims, st, st, 1, reg, 73, 0) == \
        _lib.FB_ERR_DIMENSION_MISMATCH
    assert _lib.last_error() == "Plan region is outside array dimensions."
    reg2 = (ctypes.c_int32 * 2)(2, 1)
    assert _lib.lib.fb_plan_create_nd(ctypes.byref(h), 0, -1, 2, dims, st, st, 2, reg2, 73, 0) == \
        _lib.FB_ERR_DIMENSION_MISMATCH
    assert _lib.last_error() == "Region is invalid."


def test_header_flags_match_python_constants():
    import re
    import ffta_b200 as F
    text = open(HEADER).read()
    defs = dict(re.findall(r"\b(FB_(?:FLAG|SERVER)_\w+)\s*=\s*(\d+)u?", text))
    assert "FB_SERVER_NO_GRAPHS" in defs and "FB_FLAG_TENSOR_STAGE" in defs
    for name, val in defs.items():
        assert getattr(F, name) == int(val), name
