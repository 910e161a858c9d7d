import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def built():
    """The in-tree librfd.so and liboracle.so (built on first use)."""
    import oracle
    import robotfd_b200 as rfd
    if not os.path.exists(rfd.LIB_PATH) or not os.path.exists(rfd.FD_PATH):
        rfd.build()
    oracle.lib()
    return rfd


@pytest.fixture(scope="session")
def ctx(built):
    """GPU context; raises (never skips) when no device is usable."""
    c = built.Context(0)
    yield c
    c.close()
