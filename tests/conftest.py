import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "visual-simulation-of-smoke_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def smoke_lib():
    import smoke_b200

    return smoke_b200.SmokeLibrary()


@pytest.fixture(scope="session")
def cuda_stream():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.cuda.Stream()
