import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a library)")


def has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_cuda():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def chain_scene():
    from colb_b200 import scene as S
    return S.load_npz_scene(os.path.join(GOLDEN, "chains_scene.npz"))


@pytest.fixture(scope="session")
def chain_pairs():
    return np.load(os.path.join(GOLDEN, "chains_pairs.npz"))


@pytest.fixture(scope="session")
def built_library():
    """Builds libabd_b200.so once per session (nvcc cross-compiles without a GPU)."""
    from colb_b200 import build_lib
    return build_lib.build()
