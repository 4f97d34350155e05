"""Shared test setup.

Markers: `gpu` tests need a CUDA device (B200) and run the library's kernels;
everything else runs on the CPU.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device; GPU tests fail (not skip) without one."""
    import torch
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    return torch
