"""Shared pytest configuration.

Marker ``gpu``: the test needs a CUDA GPU (B200) and the built
``hydra_b200/libhydra_casl.so``; everything else runs on CPU.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built CUDA library")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library, loaded (a GPU test fails loudly if it is missing)."""
    from hydra_b200 import casl
    return casl.load_library()
