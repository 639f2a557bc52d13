"""Shared fixtures.  `-m gpu` tests need a B200; everything else runs on CPU.

The CUDA library is built in-tree on first use (nvcc cross-compiles without a
GPU) and the oracle (the checker) with `make -C oracle`.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import __graft_entry__ as entry  # noqa: E402
import oracle_ctypes as orc  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


@pytest.fixture(scope="session")
def pkg():
    entry.build()  # incremental: recompiles only stale translation units
    return entry.load_package()


@pytest.fixture(scope="session")
def oracle():
    orc.lib()
    return orc


@pytest.fixture(scope="session")
def ctx(pkg):
    c = pkg.GpuContext.create(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def golden():
    import json
    return json.loads((ROOT / "tests" / "golden" / "reference_tables.json").read_text())


def rel_err(a, b, floor=1e-6):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)
