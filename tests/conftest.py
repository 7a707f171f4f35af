"""Shared test setup: the `gpu` marker, import paths and fixtures.

GPU tests call the CUDA library through its C ABI (the ctypes binding in
cuda-ipc-benchmarks_b200/lulesh_b200.py); the CPU oracle (oracle/) is the
checker.
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "cuda-ipc-benchmarks_b200")
ORACLE = os.path.join(REPO, "oracle")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running on the device")


@pytest.fixture(scope="session")
def lulesh():
    import lulesh_b200

    lulesh_b200.load_library()
    return lulesh_b200


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.load()
    return oracle


def rel(a: float, b: float) -> float:
    return abs(a - b) / max(abs(b), 1e-300)
