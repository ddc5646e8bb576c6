import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build the product library and the CPU oracle once per session."""
    so = os.path.join(ROOT, "fvmpor_b200", "libfvmpor_b200.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "fvmpor_b200"), "-j8"], check=True,
                       capture_output=True)
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    yield


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test requested but no CUDA device is visible")
    torch.cuda.set_device(0)
    return torch.device("cuda:0")
