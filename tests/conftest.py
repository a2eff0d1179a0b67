import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as O
    O.build()
    O.set_threads(1)   # the reference's single-thread pair and summation order
    return O


@pytest.fixture(scope="session")
def gpu_lib():
    """The in-tree sm_100a library; GPU tests fail (not skip) when it is missing."""
    from simp_b200 import build, _lib
    build.build()
    return _lib.load()
