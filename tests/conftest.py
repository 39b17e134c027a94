"""Shared test setup: import paths, the `gpu` marker and oracle fixtures.

`-m "not gpu"` tests run here without a GPU: the oracle against the
reference's own outputs, the host logic and the C ABI surface.  `-m gpu`
tests run the CUDA path through the C ABI and compare it with the oracle.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "hundun-flow_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def oracle_built():
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "libhfps_oracle.so"],
                   check=True, stdout=subprocess.DEVNULL)
    return True


@pytest.fixture(scope="session")
def cuda_library():
    """The in-tree CUDA library; builds it when missing."""
    sys.path.insert(0, os.path.join(ROOT, "hundun-flow_b200"))
    import build as hfps_build  # hundun-flow_b200/build.py
    return hfps_build.build()
