import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def ora():
    """The CPU oracle (built on first use)."""
    from oracle import oracle as o
    o.load()
    return o


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """The CUDA library; GPU tests fail (not skip) if it cannot load."""
    if not _has_gpu():
        pytest.skip("no CUDA device")
    from inmsom_elfs_b200 import build
    build.build()
    from inmsom_elfs_b200 import _lib, solver
    _lib.load()
    return solver


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """Normwise relative difference max|a-b| / max|b| (0 if both are zero)."""
    d = float(np.max(np.abs(a - b)))
    s = float(np.max(np.abs(b)))
    return d if s == 0.0 else d / s
