import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) and libexcfv.so")


@pytest.fixture(scope="session")
def gpu_fv():
    """One libexcfv handle for the GPU tests (fails loudly if the library is missing)."""
    from exciting_b200.fv import FirstVariational
    fv = FirstVariational(0)
    yield fv
    fv.close()
