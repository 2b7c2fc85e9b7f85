"""Test set-up: the gpu marker, import paths, and shared helpers.

Tests marked gpu call the CUDA library through its C ABI and compare with the
CPU oracle (oracle/); the others run on CPU only (the oracle against the
reference's own FP64 twin, host logic, and that the library loads)."""
from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def splat_module():
    """The product package (its directory name has a hyphen)."""
    return importlib.import_module("vibe-splat_b200")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def check_close(a, b, what: str, min_cosine: float, max_ratio_error: float) -> None:
    """The reference's gradient comparison (tests/test_train.cpp:38-54): direction
    by cosine and length by the ratio of norms."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    assert a.shape == b.shape, what
    aa, bb, ab = float(a @ a), float(b @ b), float(a @ b)
    assert aa > 0.0 and bb > 0.0, f"{what}: a zero vector"
    cosine, ratio = ab / np.sqrt(aa * bb), np.sqrt(aa / bb)
    print(f"  {what:24s} cosine {cosine:.6f}, length ratio {ratio:.5f}")
    assert cosine > min_cosine, f"{what}: cosine {cosine}"
    assert abs(ratio - 1.0) < max_ratio_error, f"{what}: length ratio {ratio}"


@pytest.fixture(scope="session")
def splat():
    if not cuda_available():
        pytest.skip("no CUDA device")
    return splat_module()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    return o
