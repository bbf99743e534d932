import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (str(ROOT), str(ROOT / "cuda-lbm-ibm-fvm_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


CUDA = _cuda_available()


@pytest.fixture(scope="session")
def cuda():
    if not CUDA:
        pytest.fail("GPU test selected but no CUDA device is visible")
    return True


@pytest.fixture(scope="session")
def V():
    import vof_b200

    vof_b200.lib()
    return vof_b200


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle

    oracle.oracle_lib()
    return oracle
