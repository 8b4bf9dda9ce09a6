import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libhappyray_b200.so")
    config.addinivalue_line("markers", "slow: full-size configuration (minutes on CPU)")


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
def oracle():
    import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def hrlib():
    """Build (incrementally) and load the CUDA library."""
    from happyray_b200 import build as B
    if not B.OUT.exists() or os.environ.get("HR_REBUILD"):
        B.build()
    from happyray_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def engine(hrlib):
    from happyray_b200 import Engine
    e = Engine(0)
    yield e
    e.cleanup()


@pytest.fixture(scope="session")
def c1_scene():
    from happyray_b200 import scenes as S
    return S.heightfield(129, 0)


@pytest.fixture(scope="session")
def small_clusters():
    from happyray_b200 import scenes as S
    return S.clusters(60_000, seed=3)


def as_v4(v):
    v = np.asarray(v, np.float32)
    out = np.zeros((v.shape[0], 4), np.float32)
    out[:, :3] = v
    return out
