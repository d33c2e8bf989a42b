"""Shared test setup: import paths, the `gpu` marker, and device fixtures."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "master-of-puppets_b200", ROOT / "oracle", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device")


@pytest.fixture(scope="session")
def cuda_device():
    import mopcuda
    dev = mopcuda.Device(0)
    yield dev
    dev.close()
