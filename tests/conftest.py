"""Test configuration: the ``gpu`` marker, package/oracle loaders and fixture access."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "tests"))

import __graft_entry__ as entry  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pkg():
    return entry.load_package()


@pytest.fixture(scope="session")
def oracle():
    return entry.load_oracle()


def golden(name: str):
    return np.load(GOLDEN / f"{name}.npz")


RUN_CASES = ["c1", "bh0", "bh1", "lay", "box"]
BLK_CASES = [f"blk{n}" for n in range(2, 10)]
