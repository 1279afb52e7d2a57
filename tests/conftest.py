"""pytest configuration: the ``gpu`` marker and shared fixtures.

``-m "not gpu"`` runs on any CPU host (oracle KATs, parser, C-ABI exports,
gloo multi-rank logic).  ``-m gpu`` needs a CUDA device and exercises the
product library through its C-ABI against the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libferam_gpu.so")


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib
    return oracle_lib.load()


@pytest.fixture(scope="session")
def fg():
    import feram_b200
    feram_b200.lib()
    return feram_b200
