import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_ROOT = os.path.join(REPO, "falcon-accelerate-graph-vector-search_b200")
ORACLE = os.path.join(REPO, "oracle")
for p in (PKG_ROOT, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_mod():
    import build_oracle
    build_oracle.build_oracle()
    import oracle
    return oracle


@pytest.fixture(scope="session")
def lib():
    from falcon_b200 import _lib
    return _lib.load()


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
