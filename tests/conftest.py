import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the B200 kernels)")


def pytest_collection_modifyitems(config, items):
    # GPU tests must never pass silently without a GPU: they fail loudly.
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(pytest.mark.usefixtures("require_cuda"))


@pytest.fixture
def require_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test requires a CUDA device")
