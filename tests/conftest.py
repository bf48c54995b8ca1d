import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def cuda():
    """The GPU tests run the product's CUDA kernels; without a GPU they fail
    loudly instead of passing on some fallback."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but no CUDA device is available")
    torch.cuda.init()
    return torch.device("cuda:0")
