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


def pair_digest(pairs):
    """Count and SHA-256 of an (npairs, 2) array of unordered pairs, each
    written i < j, sorted by (i, j), as little-endian int32: the full-size
    fixtures store this instead of the pairs themselves."""
    import hashlib
    import numpy as np
    p = np.asarray(pairs, np.int64).reshape(-1, 2)
    p = np.sort(p, axis=1)
    p = p[np.lexsort((p[:, 1], p[:, 0]))].astype("<i4")
    return len(p), hashlib.sha256(p.tobytes()).hexdigest()


def rms_rel(a, b):
    """RMS relative difference |a - b| / |b| over all components."""
    import numpy as np
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))
