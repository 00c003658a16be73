import importlib
import json
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")

FIELDS = ["outer", "numX", "numY", "numT", "s0", "t", "alpha", "nu", "beta"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: CPU test taking more than a few seconds")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module("futhark-benchmarks_b200")


@pytest.fixture(scope="session")
def tke():
    return importlib.import_module("futhark-benchmarks_b200.tke")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.load()
    return o


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "locvolcalib_golden.json")) as f:
        return json.load(f)["datasets"]


@pytest.fixture(scope="session")
def ctx(pkg):
    c = pkg.Context()
    yield c
    c.close()


def dataset_args(entry):
    return [entry[k] for k in FIELDS]
