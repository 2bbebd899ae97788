import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "ascend-fft_b200"
for p in (str(PKG), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("CUDA GPU required")
    return torch.device("cuda", 0)


@pytest.fixture(scope="session")
def ctx(cuda):
    import bfly
    c = bfly.Context()
    assert c.init() == 0
    yield c


@pytest.fixture(scope="session")
def plan(ctx):
    p = ctx.make_plan(ctx_default_id())
    assert p is not None
    return p


def ctx_default_id():
    import bfly
    return bfly.DEFAULT_CANDIDATE
