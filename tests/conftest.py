"""Shared fixtures. GPU tests are marked ``@pytest.mark.gpu``; everything else
runs on CPU. The oracle (oracle/) is the checker only."""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running case")


def _ensure_port():
    so = os.path.join(ROOT, "oracle", "libinlm_oracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "port"], check=True)
    return so


@pytest.fixture(scope="session")
def port():
    _ensure_port()
    from oracle.oracle import Port
    return Port()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        pytest.skip("reference CPU build (oracle/_ref) not present on this machine")
    return Reference()


@pytest.fixture(scope="session")
def lib():
    from microtomodenoise_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def golden_filter():
    return np.load(os.path.join(GOLDEN, "filter_small.npz"))


@pytest.fixture(scope="session")
def golden_noise():
    return np.load(os.path.join(GOLDEN, "noise_small.npz"))


@pytest.fixture(scope="session")
def golden_tables():
    return np.load(os.path.join(GOLDEN, "tables.npz"))


def gpu_available() -> bool:
    try:
        import ctypes
        rt = ctypes.CDLL("libcudart.so")
    except OSError:
        try:
            import torch
            return torch.cuda.is_available()
        except Exception:
            return False
    n = ctypes.c_int(0)
    return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0


@pytest.fixture(scope="session")
def gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from microtomodenoise_b200 import _lib
    _lib.load()
    return True
