"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs the oracle against the golden vectors, the host logic and
the C-ABI load/export checks on CPU; `-m gpu` runs the parity tests through
the C ABI on a B200.
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "3dfilteredbackprojection-public_b200"
for p in (ROOT / "oracle", PKG, ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


def relative_rmse(x, ref):
    import numpy as np
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.sqrt(((x - ref) ** 2).sum() / max((ref ** 2).sum(), 1e-300)))


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build(with_ref=True)  # the reference FFT is built only where its sources are present
    return O


@pytest.fixture(scope="session")
def phantoms():
    import phantoms as P
    return P


@pytest.fixture(scope="session")
def fbp():
    """The ctypes mirror over the built library (host-only calls work without a GPU)."""
    import build as B
    B.build()
    import fbp_b200
    return fbp_b200
