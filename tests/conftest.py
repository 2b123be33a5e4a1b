import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "ntt-tensorcore_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
BABYBEAR = 2013265921
Q60 = 1152921504577486849


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    return torch


def to_dev(torch, arr):
    """numpy uint32/uint64 -> CUDA tensor holding the same bytes."""
    arr = np.ascontiguousarray(arr)
    if arr.dtype == np.uint64:
        return torch.from_numpy(arr.view(np.int64)).cuda()
    if arr.dtype == np.uint32:
        return torch.from_numpy(arr.view(np.int32)).cuda()
    raise TypeError(arr.dtype)


def to_host(t, dtype):
    t = t.detach().cpu().contiguous().numpy()
    return t.view(dtype)
