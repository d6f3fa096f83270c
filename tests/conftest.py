import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (test infrastructure): built on first use."""
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def sb():
    """The product library (CUDA, no fallback)."""
    import sonium_b200
    from sonium_b200 import build

    build.build()
    return sonium_b200


def golden_path(name: str) -> str:
    return os.path.join(GOLDEN, name)
