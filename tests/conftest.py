import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100) GPU")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def native_lib():
    """The product library (built in-tree); build it if it is missing."""
    from libapsm_b200 import _native

    if not _native.LIB_PATH.exists():
        from libapsm_b200 import build

        build.build()
    return _native.load()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle

    if not oracle.ORACLE_SO.exists():
        oracle.build_oracle()
    return oracle


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no GPU in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
