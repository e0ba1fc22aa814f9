import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def restatement():
    import oracle

    return oracle.Restatement()


@pytest.fixture(scope="session")
def reference_cpu():
    import oracle

    if not oracle.ReferenceCPU.available():
        pytest.skip("reference CPU library not built (oracle/_ref); the golden fixtures still pin the oracle")
    return oracle.ReferenceCPU()
