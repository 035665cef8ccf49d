import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np
    g = np.load(os.path.join(ROOT, "tests", "golden", "das_golden.npz"))
    meta = json.loads(bytes(g["__meta__"]).decode())
    return g, meta
