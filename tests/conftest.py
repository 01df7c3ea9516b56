import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O

    O.build_oracle()
    return O


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np

    here = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(here, "golden.json")) as f:
        g = json.load(f)
    arrays = dict(np.load(os.path.join(here, "golden_small.npz")))
    return g, arrays
