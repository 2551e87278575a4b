"""Shared pytest configuration.

`gpu` marks tests that need a B200 and the built CUDA library; everything else
runs on the CPU (oracle against golden fixtures, host-side logic, library
exports, multi-process gloo paths)."""
import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libinvariantq.so")


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import Port
    return Port()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    d = REPO / "tests" / "golden"

    def load(name):
        return np.load(d / f"{name}.npz", allow_pickle=False)
    return load
