"""Test configuration.

Markers: ``gpu`` -- needs a CUDA device and the built library (run with ``-m gpu`` on a B200);
everything else runs on CPU (``-m "not gpu"``).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libannvedi_b200.so")
    config.addinivalue_line("markers", "slow: full-size property checks")


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test ran without a visible CUDA device")
    return torch.device("cuda:0")
