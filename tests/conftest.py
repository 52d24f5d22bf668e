"""Test configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs on any machine (oracle pins, ABI/layout checks, host
logic, multi-process CPU tests); `-m gpu` needs a B200 and calls the suite
through its C ABI.
"""
import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built suite libraries")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle.oracle import OracleLib
    return OracleLib()


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
