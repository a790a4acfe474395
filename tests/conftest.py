import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    import oracle
    from rtnn_b200 import build as rb
    rb.build()
    oracle.build()


_ensure_built()


@pytest.fixture(scope="session")
def ctx():
    import rtnn_b200
    c = rtnn_b200.Context(0)
    yield c
    c.close()
