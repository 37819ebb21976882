import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100) device")
    config.addinivalue_line("markers", "slow: large inputs (minutes on CPU)")


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device visible")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden_labels():
    d = np.load(os.path.join(GOLDEN, "labels.npz"))
    out = {}
    for name in d["names"]:
        name = str(name)
        out[name] = (d[f"{name}__row_ptr"], d[f"{name}__col"], d[f"{name}__labels"])
    return out


@pytest.fixture(scope="session")
def small_cases():
    from cc_mpi_b200 import graphs
    return graphs.small_cases()
