import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "optimized-gpu-accelerator_b200")
for p in (ROOT, PKG_DIR):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built engine library")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.build(reference=True)
    return O


@pytest.fixture(scope="session")
def engine_lib():
    from pramana_b200 import _lib
    return _lib.load()
