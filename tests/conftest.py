import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on a B200)")


def _ensure_lib():
    so = os.path.join(ROOT, "cudadsmc_b200", "libdsmc_b200.so")
    if not os.path.exists(so):
        from cudadsmc_b200 import build
        build.build()


_ensure_lib()


@pytest.fixture(scope="session")
def cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.init()
    return torch.device("cuda:0")
