import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def crandn(rng, shape, dtype=np.complex128):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


def cdot(a, b):
    """sum conj(a) b over all elements."""
    return np.vdot(np.asarray(a).ravel(), np.asarray(b).ravel())


def dot_err(m, Am, d, Atd):
    """|Re(<Am,d> / <m,A'd>) - 1| as ``operator/src/CudaOperator.h:190-225``, with
    <u,v> = sum u conj(v)."""
    return abs((cdot(d, Am) / cdot(Atd, m)).real - 1.0)


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
