import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the CUDA library")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import pyoracle as po

    return po.oracle_lib()


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(REPO, "tests", "golden")


@pytest.fixture(scope="session")
def ctx():
    """A library context on cuda:0; the CUDA library must load (no fallback)."""
    import sympygr_b200 as sg
    from sympygr_b200 import build

    build.build()
    c = sg.Context(0)
    yield c
    c.close()
