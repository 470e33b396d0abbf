import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_ROOT = os.path.join(REPO, "rt-dsl_b200")
for p in (REPO, PKG_ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger sizes")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test run without a visible CUDA device")
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def rtd():
    import rtdsl
    rtdsl.load()
    return rtdsl


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build()
    return oracle
