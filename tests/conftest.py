"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on a machine without a GPU: the oracle against the golden
vectors and the reference's known answers, the host-side argument logic, and
the C ABI's exports.  `-m gpu` runs the parity tests proper through the C ABI.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "ffta.jl_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
