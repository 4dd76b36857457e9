"""Shared fixtures. Tests marked `gpu` need an sm_100 device; everything else
runs on a CPU-only machine (library load, ABI, host tables, the oracle
against the reference and the golden vectors)."""
from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def grrt():
    import grrt_b200
    if not os.path.exists(grrt_b200.LIB_PATH):
        grrt_b200.build()
    grrt_b200.load_library()
    return grrt_b200


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle_bind
    oracle_bind.load_oracle(False)
    oracle_bind.load_oracle(True)
    return oracle_bind


@pytest.fixture(scope="session")
def need_gpu(grrt):
    if not grrt.cuda_available():
        pytest.skip("no sm_100 GPU")
    return True
