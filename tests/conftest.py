import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import binding
    binding.build()
    binding.set_threads(min(8, os.cpu_count() or 1))
    return binding


@pytest.fixture(scope="session")
def ctx():
    import dpa_b200
    context = dpa_b200.Context(0)
    yield context
    context.close()
