"""Shared pytest configuration.

Markers: ``gpu`` tests need a CUDA device (a B200); everything else runs on
CPU.  The package directory ``teuk-kokkos_b200`` is put on sys.path so tests
import the binding as ``teuk_b200``; the oracle bindings live in
tests/oracle_bindings.py.
"""
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO / "teuk-kokkos_b200"))
sys.path.insert(0, str(REPO / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def require_gpu():
    if not cuda_available():
        pytest.fail("GPU test collected on a host without a CUDA device")
