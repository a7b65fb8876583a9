"""Shared test set-up: import paths, the `gpu` marker, case fixtures."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "shyfemcm-ismar_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def channel():
    from shygpu import cases
    return cases.channel_case()


@pytest.fixture(scope="session")
def small3d():
    from shygpu import cases
    return cases.basin3d_case(nkn_target=1500, nlv=12)
