"""Test configuration: the `gpu` marker, import paths and shared fixtures.

Tests marked `gpu` need a B200 and call the CUDA library through its C ABI;
the rest run on CPU (oracle, host set-up, library loading and exports,
argument and table validation, multi-rank logic over gloo).
"""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "scale-dg-kernel-extraction_b200")
for p in (PKG, os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def rel_maxnorm(a, b):
    """max|a-b| / max|b|, the parity metric."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def built():
    """Builds the oracle and the library once (make is incremental)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)
    if not os.path.exists(os.path.join(PKG, "libsdg_gpu.so")):
        subprocess.run(["make", "-s", "-j8", "-C", PKG], check=True)
    return True
