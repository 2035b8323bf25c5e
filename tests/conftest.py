"""Shared test setup: import paths, the `gpu` marker, device fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "diplodocustransport.jl_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libdtb.so")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    """Skips when no CUDA device is present; on a GPU box a missing libdtb.so fails loudly."""
    if not _cuda_available():
        pytest.skip("no CUDA device")
    from dtb import _lib
    _lib.load()
    return True
