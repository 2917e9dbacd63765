import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")


def _ensure_built():
    from montepath_b200 import abi, build

    if not os.path.exists(abi.LIBRARY_PATH):
        build.build(verbose=False)
    from oracle import oracle

    oracle.build()


_ensure_built()


@pytest.fixture(scope="session")
def backend():
    from montepath_b200.backend import CudaBackend

    be = CudaBackend(0)
    yield be
    be.close()
