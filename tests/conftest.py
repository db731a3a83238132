"""Test configuration: the ``gpu`` marker selects tests that need a B200 (CUDA device)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libimps_b200.so")


@pytest.fixture(scope="session")
def ctx():
    """One library context on cuda:0 for the GPU tests (fails loudly without a device)."""
    import infinitempsalgorithms_b200 as imps
    return imps.default_context()
