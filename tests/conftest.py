import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def cuda():
    """The GPU tests run on a B200; without one they fail instead of skipping."""
    import torch

    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    from spsim_b200 import _native

    _native.use_device(torch.cuda.current_device())
    return torch.device("cuda", torch.cuda.current_device())


def golden(name):
    import numpy as np

    return np.load(os.path.join(GOLDEN, name))


def intensity_errors(I, I64, floor=1e-3):
    """(floored max relative, L2 relative) error of I against the FP64 I64."""
    import numpy as np

    I = np.asarray(I, np.float64)
    I64 = np.asarray(I64, np.float64)
    den = np.maximum(I64, floor * I64.mean())
    return float(np.max(np.abs(I - I64) / den)), float(np.linalg.norm(I - I64) / np.linalg.norm(I64))
