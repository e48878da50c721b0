import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the sm_100a kernels)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from pcbroute_b200 import build
    build.build_lib()
    build.build_oracle()
    yield


@pytest.fixture(scope="session")
def gpu():
    from pcbroute_b200 import query, _lib
    if not query.available():
        raise RuntimeError("B200 back end unavailable: " + _lib.last_error())
    return query
