"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs the CPU suite (oracle vs the reference's golden vectors,
host logic, C-ABI exports); `-m gpu` runs the parity tests of the CUDA path
through libhfgrid.so against the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hybrid-fluid-simulation_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test run without a CUDA device")
    import hfgrid
    hfgrid.init(0)
    return torch.device("cuda:0")
