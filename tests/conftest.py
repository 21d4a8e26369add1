import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (libwahgpu.so kernels)")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def unpack(d, key, i):
    o = d[key + "_off"]
    return d[key][o[i]:o[i + 1]]


@pytest.fixture(scope="session")
def gpu_ctx():
    import libfastlib_b200 as L
    ctx = L.Context(0)
    yield ctx
    ctx.close()
