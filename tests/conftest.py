import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def lib():
    from pacific_b200 import build as _b
    _b.build()
    from pacific_b200 import library
    return library()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as _o
    _o.build()
    return _o
