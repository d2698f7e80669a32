"""Shared test setup. Tests marked `gpu` need a CUDA device and the built libraries; everything
else runs on the CPU (the oracle against the golden fixtures, host logic, library exports)."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA extension")
    config.addinivalue_line("markers", "slow: long-running parity case")


def golden(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def rel_err(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def contrast_err(a, b, nm):
    """Relative error of the index contrast, as the reference's tests measure it
    (tests/test_cuda.cpp:92-97, tests/test_pipeline.cpp:19-28)."""
    a = np.asarray(a, np.float64) - nm
    b = np.asarray(b, np.float64) - nm
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="session")
def cuda():
    """torch.cuda for device buffers; skips the test without a GPU."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()
