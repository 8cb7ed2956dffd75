import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def native():
    """The native library, built in-tree if missing."""
    import glasscamerapublic_b200 as g
    if not g.LIB_PATH.exists():
        from glasscamerapublic_b200.build import build
        build()
    return g.lib()


@pytest.fixture(scope="session")
def converter(native):
    from glasscamerapublic_b200 import RawConverter
    c = RawConverter(0)
    yield c
    c.close()
