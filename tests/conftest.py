"""Shared test setup: import paths, the gpu marker, scratch directory."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "jurassic-scatter_b200")
for p in (PKG, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def workdir():
    d = os.environ.get("JSC_WORKDIR", "/tmp/jsc")
    os.makedirs(d, exist_ok=True)
    return d
