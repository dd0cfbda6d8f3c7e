"""Test configuration: the `gpu` marker and import paths.

Tests marked `gpu` need a CUDA device and the built libgcut.so; everything else runs on
the CPU (oracle, host logic, library exports, multi-process gloo tests).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cl-util_b200")
for p in (PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libgcut.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    import _gcut
    _gcut.lib()  # fails loudly when the library was not built
    return torch
