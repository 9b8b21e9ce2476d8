"""The Julia host package julia/FFTAB200 (the binding a FFTA.jl user loads).

CPU: every library entry point the package `ccall`s is declared in
include/fftab200.h and exported by libfftab200.so, and the package mirrors
FFTA's plan API (plan_fft, plan_bfft, plan_rfft, plan_brfft, mul!, *, size).
GPU: where a `julia` binary exists, the package's own parity tests
(julia/FFTAB200/test/runtests.jl, against FFTA's CPU transforms) run; the probe's
answer is the skip reason otherwise.
"""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "julia", "FFTAB200")
SRC = os.path.join(PKG, "src", "FFTAB200.jl")


def ccalled():
    return sorted(set(re.findall(r"ccall\(\(:(fb_[a-z0-9_]+),", open(SRC).read())))


def test_package_calls_only_declared_exported_symbols():
    from ffta_b200 import _lib
    header = open(os.path.join(ROOT, "include", "fftab200.h")).read()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = ccalled()
    assert {"fb_plan_create_nd", "fb_execute", "fb_execute_host", "fb_plan_destroy",
            "fb_plan_create_real", "fb_last_error"} <= set(names)
    for n in names:
        assert re.search(r"\b%s\s*\(" % n, header), n
        assert hasattr(lib, n), n


def test_package_mirrors_ffta_api():
    src = open(SRC).read()
    for pat in (r"plan_fft\(x::CuArray", r"plan_bfft\(x::CuArray", r"plan_rfft\(x::CuArray",
                r"plan_brfft\(x::CuArray", r"LinearAlgebra\.mul!\(", r"Base\.:\*\(",
                r"Base\.size\(p::GPUPlan_cx", r"No non-positive dimensions",
                r"Plan region is outside array dimensions\.", r"Region is invalid\.",
                r"only supports 1D and 2D FFTs"):
        assert re.search(pat, src), pat
    proj = open(os.path.join(PKG, "Project.toml")).read()
    assert 'name = "FFTAB200"' in proj and "AbstractFFTs" in proj and "CUDA" in proj


@pytest.mark.gpu
def test_julia_package_parity():
    jl = shutil.which("julia")
    if jl is None:
        pytest.skip("julia: not found on PATH on this host; the package's tests need Julia "
                    "with CUDA.jl and FFTA.jl")
    env = dict(os.environ, FFTAB200_LIB=os.path.join(ROOT, "ffta.jl_b200", "libfftab200.so"))
    r = subprocess.run([jl, "--project=" + PKG, "-e", "using Pkg; Pkg.test()"],
                       capture_output=True, text=True, env=env, timeout=1800)
    if r.returncode != 0 and ("not installed" in r.stderr or "Unsatisfiable" in r.stderr
                              or "could not be found" in r.stderr):
        pytest.skip("julia found, but the package's dependencies (CUDA.jl, FFTA.jl) are not "
                    "installed and there is no network: " + r.stderr[-300:])
    assert r.returncode == 0, r.stderr[-3000:]
