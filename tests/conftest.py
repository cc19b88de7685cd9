"""Test configuration: repo root on sys.path, the ``gpu`` marker, shared problem builders."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def herm(x):
    return 0.5 * (x + np.conj(np.swapaxes(x, -1, -2)))


def rand_herm(rng, shape, scale=1.0):
    a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    return scale * herm(a)


@pytest.fixture(scope="session")
def native():
    """The CUDA-backed drop-in module (GPU tests only)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cpp_hf_b200 import _native

    return _native


@pytest.fixture(scope="session")
def oracle():
    from oracle import native_np

    return native_np
