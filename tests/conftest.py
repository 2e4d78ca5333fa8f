"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on a CPU-only machine (oracle vs reference kernels and
golden fixtures, C ABI loading and argument checks); `-m gpu` runs the parity
tests through the C ABI on a CUDA device.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "janus-sim_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def root():
    return ROOT
