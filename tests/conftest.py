import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session")
def ctx():
    import torch

    import kaspan_b200 as K

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    c = K.Context(0)
    yield c
    c.close()
