"""Shared fixtures.  Tests that need a B200 are marked `gpu`; everything else
runs on the CPU (the oracle, host logic, the C ABI's symbol table)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def device():
    import droplet_b200 as dl
    d = dl.createDevice()
    yield d


@pytest.fixture(scope="session")
def renderer(device):
    import droplet_b200 as dl
    r = dl.Renderer(device)
    yield r
    r.destroy()
