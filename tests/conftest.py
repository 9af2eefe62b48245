import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "cms-julia_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def conditions():
    from pixeltrack import gen
    return gen.conditions()


@pytest.fixture(scope="session")
def event_single():
    from pixeltrack import gen
    blob, offs = gen.events(1, gen.MODE_SINGLE, ntracks=100, seed=7)
    return blob, offs


@pytest.fixture(scope="session")
def events_pu50():
    from pixeltrack import gen
    blob, offs = gen.events(4, gen.MODE_PU, pu=50, seed=11)
    return blob, offs
