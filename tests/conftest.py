"""Shared test set-up: import paths, the `gpu` marker, and the parity checkers.

Tests marked ``gpu`` need a CUDA device and call the product through its C ABI
(libcfb200.so).  Everything else runs on the CPU: the oracles against the
reference's published outputs, the host logic, and that the C-ABI library
loads and exports every symbol declared in include/cfb200.h.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cosmic-fields-lite_b200")
for p in (ROOT, os.path.join(ROOT, "oracle"), PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

os.environ.setdefault("CF_FFT_THREADS", str(min(16, os.cpu_count() or 1)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the product through its C ABI")


def _ensure_oracle():
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "all"])


_ensure_oracle()


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    return O


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "growth_and_fs_n384.npz")))
