"""Test configuration. `-m gpu` tests need a B200 and call the CUDA path through the C ABI; the rest
run on the CPU (the oracle, the host pipeline, the formats, the library's exports)."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the CUDA path through the C ABI")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the library and the oracle once (no-ops when up to date)."""
    from lightbaker_b200 import build as b
    b.build()
    import oracle
    oracle.lib()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    import lightbaker_b200 as lb
    g = lb.Gpu.new(0)
    yield g
    g.close()
