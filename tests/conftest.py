"""Test configuration: repo root on sys.path, the `gpu` marker, shared builders."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle.oracle import lib
    return lib()


@pytest.fixture(scope="session")
def cuda_lib():
    from emerge_engine_b200.build import build
    from emerge_engine_b200.abi import load_library
    build()
    return load_library()
