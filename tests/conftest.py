import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ref():
    from oracle import reflib
    if not reflib.available():
        pytest.skip("oracle/_ref/libtauref.so not built")
    return reflib


@pytest.fixture(scope="session")
def solver_factory():
    from lsms_b200 import tau
    cache = {}

    def get(lmax=3, ns=1, npola=1):
        key = (lmax, ns, npola)
        if key not in cache:
            cache[key] = tau.TauSolver(lmax, ns, npola)
        return cache[key]

    yield get
    for s in cache.values():
        s.close()
