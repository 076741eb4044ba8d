"""pytest configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs everything that needs no GPU (oracle pinning, host logic,
the C ABI's exports and argument checks); `-m gpu` runs the parity tests that
call the CUDA library through its C ABI on a B200.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def mb():
    import merle_b200
    merle_b200.lib()
    return merle_b200


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch
