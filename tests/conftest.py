"""Shared test setup: import paths, the `gpu` marker, golden fixtures."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "stencil-optimalizations_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: full-size or long-running case")


@pytest.fixture(scope="session")
def golden_cases():
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


@pytest.fixture(scope="session", autouse=True)
def _built_oracle():
    import oracle
    oracle.liboracle()
    yield
