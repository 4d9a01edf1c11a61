"""Shared fixtures of the test suite.

Tests marked `gpu` need a CUDA device and run the product through its C ABI;
everything else runs on the CPU (the oracle, host logic, symbol exports).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels through the C ABI")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle


def norm_err(a, b, floor=1e-30):
    """max |a-b| / max(max|b|, floor): the field-wide relative error used by the parity tests."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, floor)
    return float(np.max(np.abs(a - b))) / scale if a.size else 0.0
