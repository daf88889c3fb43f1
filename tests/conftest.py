"""Shared fixtures. Tests marked ``gpu`` need a CUDA device and the built library."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def golden_meta():
    import json

    return json.loads((GOLDEN / "golden.json").read_text())


@pytest.fixture(scope="session")
def golden_setup():
    return dict(np.load(GOLDEN / "setup.npz"))


@pytest.fixture(scope="session")
def golden_trajectories():
    return dict(np.load(GOLDEN / "trajectories.npz"))


@pytest.fixture(scope="session")
def golden_rooms():
    return dict(np.load(GOLDEN / "rooms.npz"))
