import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
ORACLE_DIR = os.path.join(REPO, "oracle")
if ORACLE_DIR not in sys.path:
    sys.path.insert(0, ORACLE_DIR)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) and the built libclipb.so")


def golden_config(name):
    return os.path.join(GOLDEN, "configs", name + ".txt")


def golden_npz(name):
    return os.path.join(GOLDEN, name + ".npz")


@pytest.fixture(scope="session")
def cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
