"""Shared test configuration.

Markers: `gpu` -- needs a CUDA device and the built engine (run on a B200).
Everything else runs on CPU: the oracle against the golden fixtures and
against the reference's own code (when its sources are present), host
logic, and the C ABI's exported symbols.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def engine_mod():
    import prlgt2020_b200 as P
    from prlgt2020_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    _lib.load()
    return P
