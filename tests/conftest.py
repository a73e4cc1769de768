import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# Under pytest-xdist every worker would start one OpenMP thread per core in
# the reference build and the oracle; their spinning threads then slow the
# suite from minutes to a quarter of an hour.  Each worker takes its share
# of the cores instead (set before either library loads).
if os.environ.get("PYTEST_XDIST_WORKER") and "OMP_NUM_THREADS" not in os.environ:
    _workers = max(1, int(os.environ.get("PYTEST_XDIST_WORKER_COUNT", "1")))
    os.environ["OMP_NUM_THREADS"] = str(max(1, (os.cpu_count() or 1) // _workers))



def reference_root():
    """The reference (Cardioid) checkout whose golden files the pins read:
    CARDIOID_REF, else where the oracle build found it
    (oracle/_ref/reference_root, written by oracle/ref/Makefile); an empty
    string when neither names an existing directory (the pins then skip)."""
    cand = os.environ.get("CARDIOID_REF", "")
    if not cand:
        rec = os.path.join(ROOT, "oracle", "_ref", "reference_root")
        if os.path.exists(rec):
            with open(rec) as f:
                cand = f.read().strip()
    return cand if cand and os.path.isdir(cand) else ""


REFERENCE = reference_root()


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
