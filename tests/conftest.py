"""Shared pytest setup: the `gpu` marker and device fixtures for the C-ABI tests."""
from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels through the C-ABI")


@pytest.fixture(scope="session")
def acc():
    """Initialised ACC runtime + LIBSMM on device 0, with one stream; skips without a device."""
    import libxstream_b200 as xs
    from libxstream_b200 import acc as A

    if A.ndevices() < 1:
        pytest.skip("no CUDA device")
    A.init()
    stream = A.Stream("test")
    yield A, stream
    stream.destroy()
    A.finalize()
    del xs
