import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libmps_b200.so")


def _has_gpu() -> bool:
    try:
        import torch  # noqa: F401  (only to ask whether a device exists)
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle  # oracle/oracle.py: the CPU checker
    if not os.path.exists(oracle.LIB_PATH):
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def capi():
    from mps_solvers_b200 import capi as c
    c.lib()
    return c
