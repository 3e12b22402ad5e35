import importlib
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    # libfv.so, the driver and the oracle's libraries are build products, not tracked files: build them
    # (a no-op when they are current) before any test module loads them or checks for them at
    # collection, so that a fresh checkout collects and runs every test
    importlib.import_module("neural-pde-surrogate_b200.build").build()
    from oracle import build_oracle
    build_oracle.build()


@pytest.fixture(scope="session")
def fvpkg():
    return importlib.import_module("neural-pde-surrogate_b200")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import build_oracle
    build_oracle.build_oracle()
    from oracle import oracle
    return oracle


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    return True
