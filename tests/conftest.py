"""Shared test setup.

`-m "not gpu"` tests run anywhere (oracle vs golden vectors, host logic, the
C ABI's exports); `-m gpu` tests need a CUDA device and call libxk.so.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "xrt-rs_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libxk.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.build()
    return o


@pytest.fixture(scope="session")
def golden_case():
    import json
    with open(os.path.join(GOLDEN, "diffraction_ref.json")) as f:
        return json.load(f)["test_cases"][0]


@pytest.fixture(scope="session")
def ctx():
    import xrt_rs
    c = xrt_rs.GpuContext.new()
    if c is None:
        pytest.fail("no CUDA device: -m gpu tests need a B200")
    return c
