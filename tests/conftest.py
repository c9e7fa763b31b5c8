import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_golden(name):
    import numpy as np

    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def unpack(d, prefix):
    out = []
    i = 0
    while f"{prefix}{i}" in d:
        out.append(d[f"{prefix}{i}"])
        i += 1
    return out


def deps_from(flat, offs):
    return [flat[offs[i]:offs[i + 1]].tolist() for i in range(len(offs) - 1)]


@pytest.fixture
def golden():
    return load_golden
