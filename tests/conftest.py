"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and the native library;
everything else runs on CPU (oracle, host logic, library loading)."""
from __future__ import annotations

import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the native library")


@pytest.fixture(scope="session")
def reference_vectors():
    with open(os.path.join(GOLDEN, "reference_vectors.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def config_counts():
    with open(os.path.join(GOLDEN, "config_counts.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def native_lib():
    from edge_matching_puzzle_b200 import native
    return native.load()
