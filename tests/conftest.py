import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libstratum2_b200.so")


@pytest.fixture(scope="session")
def device():
    from stratum2_b200 import Device
    d = Device(0)
    yield d
    d.close()
