import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the molla_b200 CUDA library)")


def _cuda_ok() -> bool:
    try:
        import molla_b200 as m
        e = m.Engine(0)
        e.close()
        return True
    except Exception:
        return False


@pytest.fixture(scope="session")
def engine():
    import molla_b200 as m
    e = m.Engine(0)
    yield e
    e.close()
