"""Shared fixtures. Tests marked `gpu` need a CUDA device and the built
libarcb200.so; everything else runs on the CPU (oracle, host logic, ABI load)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")
    config.addinivalue_line("markers", "slow: full-size configuration checks")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected but CUDA is not available")
    return torch


@pytest.fixture(scope="session")
def aw():
    import arcwarden_b200 as aw
    aw.load_library()
    return aw


def relerr(a, b) -> float:
    """max|a-b| / max|b| — the reference's own cross-check metric
    (tools/deposit_bench.cu:56-65)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="session")
def rel():
    return relerr
