import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def _gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this container")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def orc():
    import oracle
    if not os.path.exists(os.path.join(ROOT, "oracle", "liborc.so")):
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def qol():
    import qotential_b200 as q
    from qotential_b200 import _build
    _build.build()
    return q


def grf_apply(u, si, sj, vs, vd, ub, ubn):
    """u[i] += sum over COO entries (S - S_naive) ubn_j - (D - D_naive) ub_j,
    accumulated in COO order."""
    u = u.copy()
    np.add.at(u, si - 1, vs * ubn[sj - 1] - vd * ub[sj - 1])
    return u
