"""Shared test setup: import paths, the ``gpu`` marker, common fixtures."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "inti.jl_b200", ROOT / "oracle", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device and libinti_b200.so")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def oracle():
    import oracle as _o

    _o.lib()
    return _o


@pytest.fixture(scope="session")
def ctx():
    """The GPU context; GPU tests fail loudly (never skip to a fallback)
    when the library or the device is missing."""
    import inti_b200

    return inti_b200.default_context()


@pytest.fixture
def rng():
    return np.random.default_rng(1)
