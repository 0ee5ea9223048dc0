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


def pytest_collection_finish(session):
    """With DSMC_CHECK_FIXTURES=1, fail collection when a test asks for an
    argument that is neither a fixture nor a parameter (such a test would only
    error at setup, on the GPU box)."""
    if os.environ.get("DSMC_CHECK_FIXTURES") != "1":
        return
    missing = []
    for item in session.items:
        fi = getattr(item, "_fixtureinfo", None)
        if fi is None:
            continue
        params = getattr(getattr(item, "callspec", None), "params", {})
        for name in fi.names_closure:
            if name == "request" or name in params or fi.name2fixturedefs.get(name):
                continue
            missing.append(f"{item.nodeid}: {name}")
    if missing:
        raise pytest.UsageError("unresolved test arguments:\n" + "\n".join(missing))
