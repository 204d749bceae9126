import importlib
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on the CPU")


def load_pkg():
    return importlib.import_module("gpu-proton-dose-engine_b200")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
