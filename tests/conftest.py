import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REFERENCE = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_port():
    from oracle import port
    if not port.available():
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], check=True, capture_output=True)
    return port


@pytest.fixture(scope="session")
def cdb_lib():
    from cardioid_b200 import build, _lib
    build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def fits002():
    """BetterTT06 parameters with the shipped dt = 0.02 fits, celltype 0/1/2."""
    from cardioid_b200 import engine
    return [engine.default_params(ct, 0.02) for ct in (0, 1, 2)]
