import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
NONE_ID = 0xFFFFFFFF


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")


def load_fixture(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


SEARCH_FIXTURES = ["search_l2_d64", "search_ip_d40_int", "search_l2_d200", "search_ip_d96"]


def fixture_cases(fx):
    """(K, L) pairs stored in a search fixture."""
    out = []
    for key in fx:
        if key.startswith("ids_K"):
            k, l = key[5:].split("_L")
            out.append((int(k), int(l)))
    return sorted(out)


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    O._lib_oracle()
    return O
