"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the native libraries once (nvcc cross-compiles without a GPU)."""
    from glp_b200 import build
    build.build_all()
    yield
