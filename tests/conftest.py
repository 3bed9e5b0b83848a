import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def mpi_init():
    from tempi_b200 import mpi

    assert mpi.Init() == 0
    return mpi


@pytest.fixture(scope="session")
def cuda():
    """A GPU test's device.  On a GPU box a missing CUDA is an error, not a
    skip, so a silent fallback cannot pass."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA is not available for a test marked gpu")
    torch.cuda.init()
    return torch.device("cuda:0")
