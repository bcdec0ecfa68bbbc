"""Shared test configuration: the ``gpu`` marker, import paths and golden fixtures."""

import json
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
for p in (ROOT, ROOT / "mammos-mumag_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    return GOLDEN


@pytest.fixture(scope="session")
def cube_mesh():
    """The reference's ``tests/data/cube.fly``: 20 nm cube in a sphere shell (tags 1/2/3)."""
    g = np.load(ROOT / "mammos-mumag_b200" / "mammos_mumag" / "mesh" / "CUBE_20_nm.npz")
    return g["X"], g["T"], g["tag"].astype(np.int32)


@pytest.fixture(scope="session")
def energies():
    return json.loads((GOLDEN / "energies.json").read_text())
