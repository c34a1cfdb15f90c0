"""Shared pytest configuration.

Markers: `gpu` tests need a CUDA device and exercise libocean_b200.so through
its C ABI; everything else runs on the CPU (oracle pins, ABI layout, host-side
logic) and never launches device work.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device; calls the CUDA library")


@pytest.fixture(scope="session")
def cuda_device():
    """Fails (never skips) when a GPU test runs without a usable device or
    without the built library: those are exactly the conditions a silent
    fallback would hide."""
    import torch

    assert torch.cuda.is_available(), "gpu test needs a CUDA device"
    import oceanlib_b200 as ob

    ob.lib()  # raises if libocean_b200.so was not built
    torch.cuda.init()
    return torch.cuda.current_device()
