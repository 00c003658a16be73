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


# The reference's dataset files, byte for byte (gzip-compressed), at their
# paths in the reference tree (regenerated by tests/golden/make_golden.py).
DATASETS = os.path.join(GOLDEN, "datasets")
_GOLDEN_FILES = {
    "tridiag32_small": "misc/ocean-sim/data/tridiag32-small",
    "tke32_small": "misc/ocean-sim/data/tke32-small",
    "optionpricing_small": "finpar/OptionPricing-data/small",
    "optionpricing_medium": "finpar/OptionPricing-data/medium",
    "optionpricing_large": "finpar/OptionPricing-data/large",
}


def read_dataset(relpath):
    """The values of a reference dataset file, e.g. "finpar/LocVolCalib-data/small.in"."""
    fd = importlib.import_module("futhark-benchmarks_b200.futhark_data")
    return fd.read_file(os.path.join(DATASETS, relpath + ".gz"))


def golden_npz(name):
    """A fixture's inputs and outputs by name: in00, in01, ... and out0, out1, ...
    (the tridiagonal fixture also as a, b, c, y and x)."""
    stem = _GOLDEN_FILES[name]
    ins = read_dataset(stem + ".in")
    outs = read_dataset(stem + ".out")
    d = {f"in{i:02d}": v for i, v in enumerate(ins)}
    d.update({f"out{i}": v for i, v in enumerate(outs)})
    if name == "tridiag32_small":
        d.update(a=ins[0], b=ins[1], c=ins[2], y=ins[3], x=outs[0])
    return d
