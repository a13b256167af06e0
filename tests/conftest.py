import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libeimp_b200.so")


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
def ctx():
    from eimp_b200.engine import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def tiny():
    from eimp_b200 import synth
    return synth.generate("tiny")


@pytest.fixture(scope="session")
def smalltest():
    from eimp_b200 import synth
    return synth.generate("small-test")


def golden_path(name: str) -> str:
    return os.path.join(ROOT, "tests", "golden", name)
