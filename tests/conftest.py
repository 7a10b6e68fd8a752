import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(autouse=True)
def _biout_into_tmp(tmp_path, monkeypatch):
    """utils.biout appends to necg.out in the working directory, as the
    reference's does; point it at the test's own temporary directory."""
    from nbo_correlatedgaussians_b200 import utils
    monkeypatch.setattr(utils, "_OUTPUT_FILE", str(tmp_path / "necg.out"))
