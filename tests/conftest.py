import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden(name):
    import numpy as np
    return np.load(os.path.join(GOLDEN, name + ".npz"))
