import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libcmsgpu.so")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the oracle (CPU checker) and the CUDA library once per session."""
    from oracle import oracle as O
    O.build()
    O.set_threads(1)  # the oracle sums in the reference's single-thread order
    from cms2d_b200 import build as B
    B.build()
    yield
