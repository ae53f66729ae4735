"""Test configuration: the `gpu` marker and shared helpers.

Tests marked `gpu` need a CUDA device and call the engine through its C ABI
(libvine.so).  Everything else runs on the CPU: the oracle against the
golden vectors, the workload generators, the host logic, the ABI exports and
the multi-process (gloo) paths."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    if not oracle.ORACLE_SO.exists():
        oracle.build()
    return oracle
