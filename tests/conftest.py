"""Shared test setup: the `gpu` marker (tests that need a CUDA device, run on a B200),
the repository on sys.path, and a context fixture for GPU tests."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")


@pytest.fixture(scope="session")
def ctx():
    import luce_render_b200 as lr
    context = lr.Context(0)
    yield context
    context.close()
