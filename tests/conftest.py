"""Test configuration.

Tests marked ``gpu`` need a CUDA device (a B200) and the built library;
everything else runs on the CPU: the oracle against its known-answer tests,
the host-side logic, and the C-ABI library's exported symbols.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and libntlp_gpu.so")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    import pyoracle
    pyoracle.build()
    return pyoracle
