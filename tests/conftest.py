import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a B200); run with -m gpu")


@pytest.fixture(scope="session")
def ctx():
    """One libab2 context on cuda:0 for the GPU tests."""
    from alien_b200 import abi

    c = abi.Context(int(os.environ.get("AB2_DEVICE", "0")))
    yield c
    c.close()
