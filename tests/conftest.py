"""Shared test configuration.

``-m gpu`` tests need a CUDA device and call the engine through its C ABI;
everything else runs on the CPU (the oracle against the reference's golden
vectors, host-side logic, and that the C-ABI library loads and exports every
declared symbol).
"""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "yang-mills_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "reference_vectors.json")) as fh:
        return json.load(fh)["vectors"]


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O
