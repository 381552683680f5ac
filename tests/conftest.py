"""Test configuration: the ``gpu`` marker and shared fixtures."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def built_library():
    """Path of the in-tree C ABI library, building it when missing or stale."""
    from rcabeam_b200 import _build

    return _build.build()
