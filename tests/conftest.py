import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100) device; run with -m gpu")


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for gpu-marked tests.  Fails (does not skip) without one: a gpu
    test that cannot reach the device has not verified anything."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but torch.cuda.is_available() is False")
    from hindemith_b200 import _lib

    _lib.lib()  # the native library must load
    return torch.device("cuda:0")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def golden_files(pattern):
    return sorted(glob.glob(os.path.join(GOLDEN, pattern)))


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def assert_bitexact(a, b, what=""):
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if not np.array_equal(bits(a), bits(b)):
        diff = np.argwhere(bits(a) != bits(b))
        i = tuple(diff[0])
        raise AssertionError(f"{what}: {len(diff)} elements differ; first at {i}: "
                             f"{a[i]!r} vs {b[i]!r}; max |d| = {np.abs(a - b).max():.3g}")
