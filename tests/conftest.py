"""Shared fixtures and the `gpu` marker.

`-m "not gpu"` runs everything that needs no GPU (oracle pinning, the C-ABI
library's exports, host logic, gloo multi-process logic); `-m gpu` runs the
parity tests proper, through the C ABI of libwbfmm_b200.so on a B200.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def restatement():
    from oracle.oracle_api import Restatement
    return Restatement()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle_api import Reference, have_reference
    if not have_reference():
        pytest.skip("oracle/_ref/libwbfmm_ref.so not built (reference sources absent)")
    return Reference()


@pytest.fixture(scope="session")
def gpu_lib():
    from wbfmm_b200 import engine
    lib = engine.load_library()      # raises if the library is missing
    if engine.device_count() < 1:
        pytest.fail("no CUDA device visible to libwbfmm_b200.so")
    return lib
