import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

GOLDEN = os.path.join(ROOT, "tests", "golden")
EV = 1.60217653e-19


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and the built CUDA library")


def golden(name):
    """Load a golden text fixture (gzipped) as a float array, skipping comment lines."""
    return np.loadtxt(os.path.join(GOLDEN, name + ".txt.gz"), comments="#")


def golden_lines(name, prefix):
    import gzip
    with gzip.open(os.path.join(GOLDEN, name + ".txt.gz"), "rt") as f:
        return [l.split()[1:] for l in f if l.startswith(prefix + " ")]


@pytest.fixture(scope="session")
def oracle_halfspace():
    import pyoracle
    from cudamonsel_b200 import scenes
    sc = scenes.halfspace()
    b, h = pyoracle.build_oracle(sc)
    return b, h, sc


@pytest.fixture(scope="session")
def oracle_lines():
    import pyoracle
    from cudamonsel_b200 import scenes
    sc = scenes.lines()
    b, h = pyoracle.build_oracle(sc)
    return b, h, sc


@pytest.fixture(scope="session")
def engine():
    from cudamonsel_b200 import capi
    e = capi.Engine(0)
    yield e
    e.close()
