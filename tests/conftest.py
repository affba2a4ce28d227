"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on the CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def table():
    """Synthetic Helmholtz table (x2 layout: 541 x 201)."""
    from phlegethon_b200 import helm_table
    return helm_table.generate()


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    pyoracle.load()
    return pyoracle


@pytest.fixture(scope="session")
def gpu_lib():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test without a CUDA device")
    from phlegethon_b200 import abi
    return abi.load_library()
