import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
REFERENCE = os.environ.get("OTFWI_REF", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def lib():
    """The built CUDA library (built on first use; no fallback)."""
    from otfwi_b200 import _build, _lib
    _build.build()
    return _lib.load()


def golden(name):
    import numpy as np
    return np.load(os.path.join(GOLDEN, name))
