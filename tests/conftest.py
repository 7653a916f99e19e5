import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def ctx_factory():
    from chili_b200 import gpu
    made = []

    def make():
        c = gpu.Context(0)
        made.append(c)
        return c
    yield make
    for c in made:
        c.close()
