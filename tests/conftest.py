import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size cases")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle("oracle")


@pytest.fixture(scope="session")
def golden_kat():
    import numpy as np
    return np.load(os.path.join(GOLDEN, "kat_functions.npz"))


@pytest.fixture(scope="session")
def golden_cli():
    import json
    import numpy as np
    z = np.load(os.path.join(GOLDEN, "cli_cases.npz"))
    meta = json.loads(bytes(z["meta_json"]).decode())
    return z, meta
