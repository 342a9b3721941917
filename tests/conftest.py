"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device (a B200) and call the CUDA kernels
through the C ABI of libcoffee_b200.so; every other test runs on the CPU.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built_artifacts():
    """Build the oracle restatement and the library in-tree if they are
    missing or older than their sources (cheap no-op otherwise)."""
    import subprocess

    oracle_dir = os.path.join(ROOT, "oracle")
    lib = os.path.join(oracle_dir, "liboracle.so")
    srcs = [os.path.join(oracle_dir, f) for f in ("ffe_oracle.c", "ffe_oracle.h", "ffe_oracle_impl.h")]
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(s) for s in srcs):
        subprocess.run(["make", "-C", oracle_dir, "port"], check=True, capture_output=True)
    from coffee_b200 import build

    if os.path.exists(os.path.join(ROOT, "coffee_b200", "csrc")):
        try:
            build.build()
        except RuntimeError:
            # no nvcc on this machine: tests that need the library will say so
            pass
    yield
