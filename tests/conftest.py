import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GRAPHS = ["tiny_path7", "edge_cases", "hub", "rmat_s10_e8"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def golden_graph(name):
    d = os.path.join(GOLDEN, "graphs", name)
    adj = np.load(os.path.join(d, "adj.npz"))
    meta = json.load(open(os.path.join(d, "meta.json")))
    return d, adj["rowptr"], adj["cols"], meta


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    if not os.path.exists(oracle.LIB_PATH):
        oracle.build(ref=False)
    return oracle
