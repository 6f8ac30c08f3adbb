"""Shared pytest configuration.

Markers: ``gpu`` -- needs a CUDA device (sm_100a) and the built library.
The CPU suite (``-m "not gpu"``) covers the oracle pins, host logic and the
C-ABI surface; GPU tests call the kernels through the C ABI.
"""

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
for p in (str(ROOT),):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: requires a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def fv_golden():
    return np.load(GOLDEN / "fv_contracts.npz")


@pytest.fixture(scope="session")
def gate_golden():
    return np.load(GOLDEN / "fv_gate.npz")
