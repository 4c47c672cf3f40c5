import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")


def pytest_collection_modifyitems(config, items):
    # Order: file name order is pytest's default; nothing else to do here.
    return


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    o.build()
    return o
