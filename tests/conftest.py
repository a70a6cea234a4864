import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import piko_loader  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def pk():
    return piko_loader.load()


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    if not os.path.exists(oracle.LIB_RESTATED):
        pytest.fail("oracle/liboracle.so is not built (run make -C oracle or __graft_entry__.build())")
    return oracle


@pytest.fixture(scope="session")
def ctx(pk):
    c = pk.Context()
    yield c
    c.close()
