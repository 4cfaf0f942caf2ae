import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _reference_tree():
    """The reference tree the oracle recipe reads (OTFWI_REF overrides it);
    tests that need it skip where it is absent."""
    import subprocess
    env = os.environ.get("OTFWI_REF")
    if env:
        return env
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"],
                       capture_output=True, text=True)
    return r.stdout.strip() if r.returncode == 0 else ""


REFERENCE = _reference_tree()


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
