import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on a B200)")


@pytest.fixture(scope="session")
def native():
    """The product library (built in-tree if missing: nvcc cross-compiles without a GPU)."""
    from codag_b200 import build, native as nat

    if not nat.LIB_PATH.exists():
        build.build()
    nat.lib()
    return nat


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle_py

    oracle_py.build()
    oracle_py.lib()
    return oracle_py


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
