"""Test configuration: registers the `gpu` marker and makes sure the in-tree
library (tigerci_b200/libtigerci_sigma.so) and the oracle are built."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from tigerci_b200 import build as b

    b.build()
    from oracle import dense

    dense.build_oracle()
    yield


def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture
def need_gpu():
    if not gpu_available():
        pytest.fail("a CUDA device is required for this test (run with -m 'not gpu' on CPU)")
