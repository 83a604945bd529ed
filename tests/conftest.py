import importlib
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (HERE, ROOT, os.path.join(HERE, "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a B200)")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(HERE, "golden", "golden_proofs.json")) as f:
        return json.load(f)


def load_sgpu():
    """The product package (its directory name is not a Python identifier)."""
    return importlib.import_module("stark-swarm_b200")


@pytest.fixture(scope="session")
def sgpu():
    return load_sgpu()


@pytest.fixture(scope="session")
def ctx(sgpu):
    c = sgpu.Context(0)
    yield c
    c.close()
