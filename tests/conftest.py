import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O
    O.build()
    O.set_threads(min(4, os.cpu_count() or 1))
    return O


@pytest.fixture(scope="session")
def sp():
    import stencilparareal_b200 as S
    from stencilparareal_b200 import build
    build.build()
    return S
