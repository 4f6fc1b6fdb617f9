import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA engine")


def _cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this process")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(autouse=True)
def _env_guard(monkeypatch, tmp_path_factory):
    """Each test starts from the reference's default switches (test_eggpu_runtime.py:18-33),
    and the tuner's persisted choices go to a store of the test session, not the user's."""
    for name in ("EASYGRAPH_ENABLE_GPU", "EASYGRAPH_GPU_STRICT_ERRORS", "EASYGRAPH_CPU_PR_MAX_ITER",
                 "EASYGRAPH_CPU_PR_TOL"):
        monkeypatch.delenv(name, raising=False)
    monkeypatch.setenv("EGPR_TUNE_CACHE", str(tmp_path_factory.getbasetemp() / "tuning.txt"))
    yield
