import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through the C ABI")
    config.addinivalue_line("markers", "slow: large-n parity (minutes)")
    # build the in-tree libraries if a fresh checkout lacks them
    for d, so in (("oracle", "liboracle.so"), ("qoa_b200", "libqoa_cuda.so")):
        if not os.path.exists(os.path.join(ROOT, d, so)):
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, d)], check=True)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
