import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def ref_lib(oracle_lib):
    r = oracle_lib.ref()
    if r is None:
        pytest.skip("reference kernels (oracle/_ref) not built")
    return r


@pytest.fixture(scope="session")
def ctx():
    from incohautocorrelate_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


@pytest.fixture
def rng():
    return np.random.default_rng(12345)
