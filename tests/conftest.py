"""Test configuration: the `gpu` marker (tests that need a B200) and the builds they use.

`-m "not gpu"` runs on any machine: the oracle against its golden vectors and the reference, the host logic, and
that the C-ABI library loads and exports what include/ballasim_b200.h declares. `-m gpu` runs the parity tests
through the C ABI on a B200.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (compute capability 10.x) and the built CUDA library")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def oracle_port():
    from oracle.oracle import Port

    Port.lib()
    return Port


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import Ref

    if not Ref.available():
        pytest.skip("the reference harness is not built here (no reference tree, no prebuilt oracle/_ref)")
    return Ref


@pytest.fixture(scope="session")
def cuda_lib():
    from ballasim_b200 import _lib
    from ballasim_b200.build import build

    build()
    L = _lib.lib()
    if not L.bs_cuda_available():
        pytest.fail("no B200 visible: the gpu tests need one (they never fall back to the CPU)")
    return L
