import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (run with -m gpu)")


@pytest.fixture(scope="session")
def near_tables():
    """{case: (h, k, {(a,b,c): 9 complex})} from tests/golden/near_tensors.json."""
    with open(os.path.join(HERE, "golden", "near_tensors.json")) as f:
        raw = json.load(f)
    out = {}
    for name, c in raw.items():
        table = {}
        for row in c["tensors"]:
            v = tuple(int(t) for t in row[:3])
            vals = np.array(row[3:], dtype=np.float64)
            table[v] = vals[0::2] + 1j * vals[1::2]
        out[name] = (c["h"], c["k"], table)
    return out


@pytest.fixture(scope="session")
def reference_golden():
    with open(os.path.join(HERE, "golden", "reference_golden.json")) as f:
        return json.load(f)
