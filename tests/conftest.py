import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the oracle (CPU) once per session; the CUDA library is built by
    __graft_entry__.build() and only loaded by gpu tests."""
    from oracle import oracle
    oracle.build()
    yield
