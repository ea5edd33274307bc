"""The C++ facade on the GPU: a LinesOnLayers-style driver compiled against include/cudamonsel_b200.hpp
(tests/facade/lines_driver.cpp) gives exactly the tallies of the same scene built through the C ABI with
the same seeds (FP32 and FP64), and the program touching the rest of the facade's API runs."""
import os
import subprocess

import numpy as np
import pytest

from test_facade_cpu import ROOT, compile_driver

pytestmark = pytest.mark.gpu

FP64, FP32 = 0, 1


@pytest.fixture(scope="module")
def drivers(tmp_path_factory):
    d = tmp_path_factory.mktemp("facade")
    return {name: compile_driver(os.path.join(ROOT, "tests", "facade", name + ".cpp"), str(d / name))
            for name in ("lines_driver", "api_surface")}


def driver_scene():
    """The driver's scene through the scene recorder, with the driver's arithmetic for every length and
    its PMMA composition (elements in the order it lists them, C O H, weight fractions n_i A_i / sum)."""
    import math
    from cudamonsel_b200 import data, scenes
    nm = 1e-9
    s = scenes.SceneSpec()
    vac = scenes.vacuum(s)
    si = scenes.silicon(s)
    Z = [6, 8, 1]
    A = [data.atomic_weight(z) for z in Z]
    moles = [5.0, 2.0, 8.0]
    tot = 0.0
    for n, a in zip(moles, A):
        tot += n * a
    wf = [n * a / tot for n, a in zip(moles, A)]
    pmat = s.material(Z, A, wf, 1190.0, scenes.eV(5.5), scenes.eV(-5.5 + 5.0), scenes.eV(5.0))
    pm = s.msm(pmat)
    s.nistmott(pm, 1)
    s.fitted(pm, scenes.eV(65.4), scenes.eV(45.0))
    s.polaron(pm, 2.0e7, 1.0 / scenes.eV(4.0))
    s.csd_jln(pm, scenes.eV(45.0))
    chamber = s.region(None, vac, s.sphere([0.0, 0.0, 0.0], 0.1))
    s.region(chamber, si, s.planes([0.0, 0.0, -1.0], [0.0, 0.0, 0.0]))
    th = 3.0 * math.pi / 180.0
    for i in range(3):
        ln = s.line(-100.0 * nm, 40.0 * nm, 1000.0 * nm, th, th, 0.0, 0.0)
        s.translate(ln, [(i - (3 - 1) / 2.0) * 200.0 * nm, 0.0, 0.0])
        s.region(chamber, pm, ln)
    return scenes.Scene(s, chamber)


@pytest.mark.parametrize("prec", [FP32, FP64], ids=["fp32", "fp64"])
def test_driver_equals_c_abi(drivers, prec):
    from cudamonsel_b200 import capi, data, scenes
    npix, ntraj, seed = 6, 400, 1234
    args = [drivers["lines_driver"], data.SI_TABLES, str(npix), str(ntraj), str(seed)] + (["fp64"] if prec == FP64
                                                                                          else [])
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    rows = [l.split() for l in r.stdout.splitlines()]
    back_f = np.array([[int(x) for x in w[1:]] for w in rows if w[0] == "back"])
    yields_f = np.array([[float(w[2]), float(w[3])] for w in rows if w[0] == "pixel"])
    assert back_f.shape == (npix, 52)
    e = capi.Engine(0)
    h = scenes.build_engine(driver_scene(), e)
    nm = 1e-9
    for p in range(npix):
        xnm = (p - (npix - 1) / 2.0) * 1.0
        c = [[xnm * nm, 0.0, -100.0 * nm - 20.0 * nm]]
        b, f, st = e.run(h["chamber"], c, scenes.eV(500.0), ntraj, 50, 1.0 * nm, seed + p, precision=prec)
        assert np.array_equal(b[0], back_f[p]), p
        bse, se = scenes.yields(b, ntraj, 500.0, 50)
        assert abs(bse[0] - yields_f[p, 0]) < 1e-8 and abs(se[0] - yields_f[p, 1]) < 1e-8
    e.close()
    print("pixels %d x %d trajectories: identical tallies; BSE %s SE %s" % (
        npix, ntraj, np.round(yields_f[:, 0], 3), np.round(yields_f[:, 1], 3)))


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_api_surface_runs(drivers, prec):
    r = subprocess.run([drivers["api_surface"]] + ([prec] if prec == "fp64" else []), capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    w = r.stdout.split()
    print(r.stdout.strip())
    assert w[0] == "bins" and int(w[1]) == 80
    assert int(w[3]) > 0 and int(w[7]) >= int(w[3]) + int(w[5])  # the angle histograms count every escape
