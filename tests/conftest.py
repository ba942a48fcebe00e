"""Test configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a CUDA device (B200, sm_100a); everything else runs
on the CPU. The reference oracle (oracle/_ref/libfvmref.so, built by
`make -C oracle`) is the checker for parity tests.
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
def fvm_lib():
    from fvm_b200 import _lib

    return _lib.load()


@pytest.fixture(scope="session")
def refo():
    from oracle import ref

    if not ref.available():
        pytest.skip("reference oracle library not built (make -C oracle)")
    return ref
