import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libwrfgpu.so")


@pytest.fixture(scope="session")
def cuda_ready():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_gpu_b200 import build

    build.build()
    return True
