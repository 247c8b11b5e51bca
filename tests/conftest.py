import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build(with_ref=oracle.ref_tree_present() and not oracle.ref_available())
    return oracle


@pytest.fixture(scope="session")
def roift():
    import roift_b200
    from roift_b200 import build
    if os.path.isdir("/usr/local/cuda") and os.path.exists("/usr/local/cuda/bin/nvcc"):
        build.build()
    return roift_b200
