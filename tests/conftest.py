"""Test configuration: the `gpu` marker and the CPU oracle build.

Tests marked `gpu` need a CUDA device and the built libsalmon_b200.so; every
other test runs on the CPU.  The oracle libraries are (re)built once per
session by oracle/Makefile (the reference-derived _ref library only where the
reference tree exists; elsewhere the prebuilt copy is used if present)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    from oracle import oracle as O
    O.build()
    yield


@pytest.fixture(scope="session")
def cuda_lib():
    """The CUDA library, built for sm_100a; GPU tests fail (not skip) without it."""
    from salmon_b200 import build
    build.build()
    from salmon_b200 import _lib
    return _lib.lib()
