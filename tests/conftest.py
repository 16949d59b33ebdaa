"""Test configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a CUDA device and the in-tree library; everything
else runs on the CPU (symbolic analysis through the C-ABI, the oracle against
the reference and the golden fixtures, the host-side plan checks).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the compiled library")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the library and the checkers once per session (no-op when current)."""
    from tensors_b200 import build as tb_build
    import oracle

    tb_build.build()
    oracle.build()  # the reference target is skipped by its recipe when no checkout is present
    yield


@pytest.fixture
def rng():
    return np.random.default_rng(0x5EED0000)


def relative_residual(A, X, B):
    """||B - A X|| / (||A|| ||X|| + ||B||) in the Frobenius / 1-norms."""
    import scipy.sparse.linalg as spla

    S = A.to_scipy()
    R = B - S @ X
    nA = spla.norm(S, 1)
    return float(np.linalg.norm(R) / (nA * np.linalg.norm(X) + np.linalg.norm(B)))
