import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu on a B200)")


@pytest.fixture(scope="session")
def ctx():
    import torch

    import radix_b200 as rb
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return rb.default_context(0)
