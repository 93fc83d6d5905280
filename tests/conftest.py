import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the native library")
    config.addinivalue_line("markers", "slow: long-running parity histories")


def pytest_collection_modifyitems(config, items):
    # GPU tests are selected with -m gpu; without a GPU they are skipped
    # rather than failing, so the CPU suite stays green everywhere.
    try:
        import torch  # noqa: F401
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
