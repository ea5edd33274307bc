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


def shapes2_scene(fixes=0):
    """The shapes of the second shapes fixture: NormalCylindricalShape, NormalUnionShape and
    NShapes::createLine with rounded corners."""
    from cudamonsel_b200 import scenes
    s = scenes.SceneSpec()
    s.options = fixes
    cyl = s.cylinder([-20e-9, -10e-9, 30e-9], [25e-9, 15e-9, 50e-9], 12e-9)
    cyly = s.cylinder([10e-9, -500e-9, -30e-9], [10e-9, 500e-9, -30e-9], 8e-9)
    c, hh = (5e-9, -3e-9, 12e-9), (15e-9, 10e-9, 5e-9)
    n, p = [], []
    for a in range(3):
        for sg in (-1, 1):
            nn = [0.0, 0.0, 0.0]
            pp = list(c)
            nn[a] = float(sg)
            pp[a] += sg * hh[a]
            n += nn
            p += pp
    block = s.planes(n, p)
    cylb = s.cylinder([-20e-9, -10e-9, 30e-9], [25e-9, 15e-9, 50e-9], 12e-9)
    uni = s.union(block, cylb)
    th = 3 * 3.14159265358979323846 / 180
    rline = s.line(-100e-9, 40e-9, 1e-6, th, th, 5e-9, 8e-9)
    cylt = s.cylinder([-20e-9, -10e-9, 30e-9], [25e-9, 15e-9, 50e-9], 12e-9)
    s.translate(cylt, [30e-9, 0.0, -10e-9])
    return s, [cyl, cyly, uni, rline, cylt]


def rotate_scene():
    """The shapes of the rotated-shapes fixture (ITransform::rotate): a 6-plane block rotated by Euler angles
    about a pivot, the same block rotated with phi = 0, a tilted half-space, a cylinder rotated once (the
    rotation normalises the reference's cylinder axis) and a cylinder rotated twice."""
    from cudamonsel_b200 import scenes
    s = scenes.SceneSpec()

    def block():
        c, hh = (5e-9, -3e-9, 12e-9), (15e-9, 10e-9, 5e-9)
        n, p = [], []
        for a in range(3):
            for sg in (-1, 1):
                nn = [0.0, 0.0, 0.0]
                pp = list(c)
                nn[a] = float(sg)
                pp[a] += sg * hh[a]
                n += nn
                p += pp
        return s.planes(n, p)

    piv0, piv1, piv2, piv3 = [3e-9, -2e-9, 10e-9], [-4e-9, 6e-9, 0.0], [10e-9, 0.0, 0.0], [0.0, 5e-9, 20e-9]
    b0 = block()
    s.rotate(b0, piv0, 0.7, 0.4, -1.1)
    b1 = block()
    s.rotate(b1, piv1, 0.0, 0.9, 0.3)
    hs = s.planes([0.0, 0.0, -1.0], [0.0, 0.0, 0.0])
    s.rotate(hs, piv2, 0.2, 0.3, 0.0)
    e0, e1 = [-20e-9, -10e-9, 30e-9], [25e-9, 15e-9, 50e-9]
    c0 = s.cylinder(e0, e1, 12e-9)
    s.rotate(c0, piv3, -0.5, 1.2, 0.8)
    c1 = s.cylinder(e0, e1, 9e-9)
    s.rotate(c1, piv3, 0.0, 0.5, 0.0)
    s.rotate(c1, piv0, 1.3, -0.2, 0.6)
    return s, [b0, b1, hs, c0, c1]

