import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built engine library")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def require_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def exact_equal(a, b) -> bool:
    """Value equality (NaNs equal, +0 == -0) of two arrays of the same dtype."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f":
        return bool(np.array_equal(a, b, equal_nan=True))
    return bool(np.array_equal(a, b))


def first_mismatch(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    bad = np.nonzero(~((a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a != b)))[0]
    if a.dtype.kind != "f":
        bad = np.nonzero(a != b)[0]
    if bad.size == 0:
        return None
    i = int(bad[0])
    return dict(index=i, a=a[i], b=b[i], count=int(bad.size))
