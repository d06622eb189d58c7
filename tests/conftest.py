"""pytest configuration: the `gpu` marker, import paths, shared fixtures.

`-m "not gpu"` runs on any CPU box: the oracle against the golden vectors and the
reference engine, host logic, and the C ABI's load/export surface.
`-m gpu` runs the parity tests proper through the C ABI on a B200.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

TESTS = Path(__file__).resolve().parent
ROOT = TESTS.parent
sys.path.insert(0, str(TESTS))
sys.path.insert(0, str(ROOT))

from pkg_loader import load_package, load_submodule  # noqa: E402

GOLDEN = TESTS / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU; runs the CUDA engine")


@pytest.fixture(scope="session")
def ce():
    return load_package()


@pytest.fixture(scope="session")
def wl():
    return load_submodule("workloads")


@pytest.fixture(scope="session")
def engine(ce):
    e = ce.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="session")
def golden_ch4():
    return dict(np.load(GOLDEN / "ch4_ref.npz"))


@pytest.fixture(scope="session")
def golden_h2o():
    return dict(np.load(GOLDEN / "h2o_ref.npz"))


@pytest.fixture(scope="session")
def golden_mixed():
    return dict(np.load(GOLDEN / "mixed_ref.npz"))
