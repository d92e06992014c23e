"""Test configuration: the `gpu` marker and in-tree builds of the libraries.

CPU tests (-m "not gpu") cover the oracle against the reference's golden
vectors, host logic and the C-ABI symbol table; GPU tests (-m gpu) are the
parity tests of the CUDA path through the C ABI.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")
    oracle_lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(oracle_lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


@pytest.fixture(scope="session")
def cuda_lib():
    """The built CUDA library (built here if missing; nvcc cross-compiles)."""
    from mantlepar_b200 import build
    build.build()
    from mantlepar_b200 import _capi
    return _capi.lib()
