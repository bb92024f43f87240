import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ctx():
    from gascoignelib_b200.build import build_library
    from gascoignelib_b200.native import Context
    build_library()
    c = Context(0)
    yield c
    c.close()
