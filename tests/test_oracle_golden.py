"""Pin the C oracle (oracle/cm_oracle.c) to golden vectors dumped from the
reference's own compiled code (tests/golden/make_golden.py).

Every per-function check is bit-exact: the oracle keeps the reference's
operation order and both are compiled for x86-64 without FMA contraction.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import EV, golden, golden_lines

D = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))


def exact(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    return same.all(), np.where(~same)[0][:5]


@pytest.mark.parametrize("Z", [1, 6, 8, 14])
def test_nistmott_sigma_and_angle(oracle_lines, Z):
    """NISTMottRS::totalCrossSection / randomScatteringAngle (JMONSEL/NISTMottRS.cu:103-154),
    including the Browning branch below 50 eV and the screened Rutherford branch from 20 keV."""
    import pyoracle as po
    b, h, _ = oracle_lines
    g = golden("nistmott")
    rows = g[g[:, 0] == Z]
    if Z == 14:
        rows = rows  # Si is loaded by the lines scene too
    n = len(rows)
    sig, th = np.zeros(n), np.zeros(n)
    nd = np.zeros(n, dtype=np.int32)
    u = np.ascontiguousarray(rows[:, 2:4])
    E = np.ascontiguousarray(rows[:, 1])
    b.L.cmo_eval_nistmott(b.h, Z, n, po.dp(E), po.dp(u), D(sig), D(th), nd.ctypes.data_as(C.POINTER(C.c_int)))
    ok, bad = exact(sig, rows[:, 4])
    assert ok, bad
    ok, bad = exact(th, rows[:, 5])
    assert ok, bad
    assert (nd == rows[:, 6]).all()


@pytest.mark.parametrize("method", [2, 3])
@pytest.mark.parametrize("Z", [1, 6, 8, 14])
def test_nistmott_methods_2_3(oracle_lines, method, Z):
    """NISTMottRS::Factory100 (method 2: Browning below 100 eV) and Factory100Lin (method 3: cross section
    linear in energy below 100 eV, Browning angles), JMONSEL/NISTMottRS.cu:76-119 and :484-512."""
    import pyoracle as po
    b, h, _ = oracle_lines
    g = golden("nistmott23")
    rows = g[(g[:, 0] == method) & (g[:, 1] == Z)]
    n = len(rows)
    assert n > 400
    sig, th = np.zeros(n), np.zeros(n)
    nd = np.zeros(n, dtype=np.int32)
    u = np.ascontiguousarray(rows[:, 3:5])
    E = np.ascontiguousarray(rows[:, 2])
    b.L.cmo_eval_nistmott_method(b.h, Z, method, n, po.dp(E), po.dp(u), D(sig), D(th),
                                 nd.ctypes.data_as(C.POINTER(C.c_int)))
    ok, bad = exact(sig, rows[:, 5])
    assert ok, bad
    ok, bad = exact(th, rows[:, 6])
    assert ok, bad
    assert (nd == rows[:, 7]).all()


def test_nu_table_interpolation(oracle_halfspace):
    """NUTableInterpolation::interpolate on all four Si tables, inside and outside the domain."""
    import pyoracle as po
    b, h, _ = oracle_halfspace
    g = golden("nutable")
    for t in range(4):
        rows = g[g[:, 0] == t]
        x = np.ascontiguousarray(rows[:, 1:4])
        out = np.zeros(len(rows))
        order = int(rows[0, 4])
        b.L.cmo_eval_table(b.h, t, len(rows), po.dp(x), order, D(out))
        ok, bad = exact(out, rows[:, 5])
        assert ok, (t, bad)


def test_tabulated_inelastic(oracle_halfspace):
    """TabulatedInelasticSM (Si, methodSE 3, offset 13.54 eV): rate, PE energy loss and
    deflection, SE generation (core level, single electron, plasmon), deviate count."""
    import pyoracle as po
    b, h, _ = oracle_halfspace
    rows = golden("tabinel")
    inp = np.ascontiguousarray(rows[:, 0:9])
    out = np.zeros((len(rows), 9))
    b.L.cmo_eval_tabulated(b.h, h["si"], 1, len(rows), po.dp(inp), D(out))
    for k in range(9):
        ok, bad = exact(out[:, k], rows[:, 9 + k])
        assert ok, (k, bad)
    # the set exercises every branch
    assert rows[:, 13].sum() > 100 and (rows[:, 13] == 0).sum() > 100


@pytest.mark.parametrize("mat", [0, 1])
def test_selectable_elastic(oracle_lines, mat):
    """SelectableElasticSM for Si (one element) and PMMA (H, O, C in the reference's set order)."""
    import pyoracle as po
    b, h, _ = oracle_lines
    g = golden("elastic")
    rows = g[g[:, 0] == mat]
    inp = np.ascontiguousarray(rows[:, 1:8])
    out = np.zeros((len(rows), 5))
    b.L.cmo_eval_elastic(b.h, h["si"] if mat == 0 else h["pmma"], 0, len(rows), po.dp(inp), D(out))
    for k, col in ((0, 8), (1, 9), (2, 10), (3, 11), (4, 12)):
        ok, bad = exact(out[:, k], rows[:, col])
        assert ok, (k, bad)


def test_pmma_csd_and_rates(oracle_lines):
    """JoyLuoNieminenCSD::compute (incl. recursive halving), FittedInelSM and polaron rates."""
    import pyoracle as po
    b, h, _ = oracle_lines
    rows = np.array([[float(x) for x in l] for l in golden_lines("pmma", "csd")])
    inp = np.ascontiguousarray(rows[:, 0:2])
    out = np.zeros((len(rows), 3))
    b.L.cmo_eval_pmma(b.h, h["pmma"], len(rows), po.dp(inp), D(out))
    for k in range(3):
        ok, bad = exact(out[:, k], rows[:, 2 + k])
        assert ok, (k, bad)


def test_pmma_composition_order():
    """The PMMA element order and weight fractions the scenes use are the reference's."""
    from cudamonsel_b200 import data, scenes
    order = [int(x) for x in golden_lines("pmma", "order")[0]]
    assert tuple(order) == scenes.PMMA_Z
    wf = {int(l[0]): (float(l[1]), float(l[2])) for l in golden_lines("pmma", "wf")}
    for z, w in zip(scenes.PMMA_Z, scenes.PMMA_WF):
        assert wf[z][0] == w
        assert wf[z][1] == data.atomic_weight(z)


def test_phonon():
    """GanachaudMokraniPhononInelasticSM rate and scatter (both angle formulas)."""
    import pyoracle as po
    from cudamonsel_b200 import scenes
    s = scenes.SceneSpec()
    m = scenes.silicon(s, phonon=True)
    sc = scenes.Scene(s, m, si=m)
    b, h = po.build_oracle(sc)
    rows = golden("phonon")
    inp = np.ascontiguousarray(rows[:, 0:5])
    out = np.zeros((len(rows), 6))
    b.L.cmo_eval_phonon(b.h, h["si"], 2, len(rows), po.dp(inp), D(out))
    for k in range(6):
        ok, bad = exact(out[:, k], rows[:, 5 + k])
        assert ok, (k, bad)


def test_shapes():
    """NormalMultiPlaneShape (half-space, 6-plane block) and NormalIntersectionShape trapezoid
    lines (NShapes::createLine, translated and not): first normal, u, containment."""
    import pyoracle as po
    from cudamonsel_b200 import scenes
    s = scenes.SceneSpec()
    half = s.planes([0, 0, -1.0], [0, 0, 0])
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
    th = 3 * 3.14159265358979323846 / 180
    line = s.line(-100e-9, 40e-9, 1e-6, th, th)
    s.translate(line, [25e-9, 0, 0])
    line0 = s.line(-100e-9, 40e-9, 1e-6, th, th)
    b = po.OracleBackend()
    res = scenes.replay(s, b)
    handles = [res[half.idx], res[block.idx], res[line.idx], res[line0.idx]]
    g = golden("shapes")
    for k, sh in enumerate(handles):
        rows = g[g[:, 0] == k]
        p01 = np.ascontiguousarray(rows[:, 1:7])
        out = np.zeros((len(rows), 6))
        b.L.cmo_eval_shape(b.h, sh, len(rows), po.dp(p01), D(out))
        for j in range(5):
            ok, bad = exact(out[:, j], rows[:, 7 + j])
            assert ok, (k, j, bad)
        assert np.isfinite(rows[:, 10]).sum() > 10  # crossings exist


@pytest.mark.parametrize("fixes", [0, 1])
def test_shapes2(fixes):
    """NormalCylindricalShape (oblique, along y, translated), NormalUnionShape(block, cylinder) and
    the rounded createLine: first normal, u, contains(p0), contains(p0, p1).  The reference's
    cylinder normalises its axis by a length not yet initialised (read as 0): pinned by cases
    0-4; cases 5-7 are the reference's cylinders with the axis normalised, which the oracle
    builds with the fixes option."""
    import pyoracle as po
    from cudamonsel_b200 import scenes
    from conftest import shapes2_scene
    s, shapes = shapes2_scene(fixes)
    b = po.OracleBackend()
    res = scenes.replay(s, b)
    g = golden("shapes2")
    cases = range(5) if fixes == 0 else range(5, 8)
    for k in cases:
        sh = shapes[k if fixes == 0 else k - 5]
        rows = g[g[:, 0] == k]
        p01 = np.ascontiguousarray(rows[:, 1:7])
        out = np.zeros((len(rows), 6))
        b.L.cmo_eval_shape(b.h, res[sh.idx], len(rows), po.dp(p01), D(out))
        for j in range(6):
            ok, bad = exact(out[:, j], rows[:, 7 + j])
            assert ok, (k, j, bad)


def test_rotate():
    """ITransform::rotate of plane sets and cylinders (Utility/Transform3D.cu, NormalMultiPlaneShape.cu:257-261,
    NormalCylindricalShape.cu:324-330): first normal, u, contains(p0), contains(p0, p1) of the rotated shapes
    equal the reference's bit for bit."""
    import pyoracle as po
    from cudamonsel_b200 import scenes
    from conftest import rotate_scene
    s, shapes = rotate_scene()
    b = po.OracleBackend()
    res = scenes.replay(s, b)
    g = golden("rotate")
    for k, sh in enumerate(shapes):
        rows = g[g[:, 0] == k]
        assert len(rows) == 3000
        p01 = np.ascontiguousarray(rows[:, 1:7])
        out = np.zeros((len(rows), 6))
        b.L.cmo_eval_shape(b.h, res[sh.idx], len(rows), po.dp(p01), D(out))
        for j in range(6):
            ok, bad = exact(out[:, j], rows[:, 7 + j])
            assert ok, (k, j, bad)


def test_barrier(oracle_halfspace):
    """ExpQMBarrierSM (classical) on the vacuum/Si surface, both directions, above and
    below the 3.75 eV barrier."""
    import pyoracle as po
    b, h, _ = oracle_halfspace
    rows = golden("barrier")
    for d in (0, 1):
        r = rows[rows[:, 0] == d]
        frm, to = (h["si_region"], h["chamber"]) if d == 0 else (h["chamber"], h["si_region"])
        inp = np.ascontiguousarray(r[:, 1:7])
        out = np.zeros((len(r), 7))
        b.L.cmo_eval_barrier(b.h, frm, to, 0, len(r), po.dp(inp), D(out))
        for k in range(6):
            ok, bad = exact(out[:, k], r[:, 7 + k])
            assert ok, (d, k, bad)
        region = np.where(out[:, 6] == h["si_region"], 1, 0)
        assert (region == r[:, 13]).all()


def test_beam_hist_freepath(oracle_halfspace):
    """GaussianBeam::createElectron, Histogram::bin (insertion-point quirk), randomMeanPathLength."""
    import pyoracle as po
    b, h, _ = oracle_halfspace
    beam = np.array([[float(x) for x in l] for l in golden_lines("misc", "beam")])
    out = np.zeros((len(beam), 3))
    b.L.cmo_eval_beam(len(beam), po.dp(np.ascontiguousarray(beam[:, 0:6])), D(out))
    ok, bad = exact(out, beam[:, 6:9])
    assert ok, bad
    for l in golden_lines("misc", "hist"):
        mn, mx, nb, v, ref = float(l[0]), float(l[1]), int(l[2]), float(l[3]), int(l[4])
        assert b.L.cmo_hist_bin(mn, mx, nb, v) == ref
    fp = np.array([[float(x) for x in l] for l in golden_lines("misc", "fpath")])
    out = np.zeros(len(fp))
    b.L.cmo_eval_freepath(b.h, h["si"], len(fp), po.dp(np.ascontiguousarray(fp[:, 0:2])), D(out))
    ok, bad = exact(out, fp[:, 2])
    assert ok, bad


def _ref_runs(kind="back"):
    import os
    from conftest import GOLDEN
    runs = []
    for line in open(os.path.join(GOLDEN, "run_halfspace_1keV.txt")):
        w = line.split()
        if w and w[0] == kind:
            runs.append(np.array([int(x) for x in w[1:]]))
    return np.array(runs)


def test_whole_run_matches_reference(oracle_halfspace):
    """Whole trajectories: 1 keV pencil beam on flat Si, 4 x 10 000 primaries from the
    reference vs 2 x 10 000 from the oracle (different random streams).  BSE and SE
    yields agree within 3 standard errors and the escape spectra pass a chi-squared test."""
    import pyoracle as po
    from cudamonsel_b200 import scenes
    from cudamonsel_b200.stats import compare_spectra, yield_z
    ref = _ref_runs()
    assert ref.shape == (4, 102)
    b, h, _ = oracle_halfspace
    orc = []
    for seed in (101, 102):
        t = b.s.run(h["chamber"], 0.0, scenes.eV(1000.0), [0, 0, -20e-9], 10000, seed, 100)
        orc.append(np.array(t.back[:102]))
    orc = np.array(orc)
    z_bse, z_se = yield_z(ref.sum(0), 40000, orc.sum(0), 20000, 1000.0, 100)
    assert abs(z_bse) < 3 and abs(z_se) < 3, (z_bse, z_se)
    p = compare_spectra(ref.sum(0), 40000, orc.sum(0), 20000)
    assert p > 1e-3, p


def test_angle_histograms_match_reference(oracle_halfspace):
    """BackscatterStats' elevation (Histogram(0, pi, 180)) and azimuthal (Histogram(0, 2 pi, 360))
    histograms, BackscatterStats.cu:105-106,147-165: 1 keV pencil beam on flat Si, reference 4 x 10 000
    primaries vs oracle 2 x 10 000.  Every escape is counted once in each; the spectra pass a
    chi-squared test."""
    from cudamonsel_b200 import scenes
    from cudamonsel_b200.stats import compare_spectra
    rel, raz, rback = _ref_runs("elev"), _ref_runs("azim"), _ref_runs("back")
    assert rel.shape == (4, 182) and raz.shape == (4, 362)
    # the angles count every escape; the energy histogram misses those whose bin falls past its overflow slot
    assert (rel.sum(1) == raz.sum(1)).all() and (rel.sum(1) >= rback.sum(1)).all()
    assert (rel.sum(1) - rback.sum(1) < 0.01 * rel.sum(1)).all()
    assert rel[:, :92].sum() == 0  # a half-space only back-scatters: elevation >= pi/2
    b, h, _ = oracle_halfspace
    oel, oaz = [], []
    for seed in (101, 102):
        t = b.s.run(h["chamber"], 0.0, scenes.eV(1000.0), [0, 0, -20e-9], 10000, seed, 100)
        oel.append(np.array(t.elevation[:]))
        oaz.append(np.array(t.azimuth[:]))
        assert sum(t.elevation) == sum(t.azimuth) == sum(t.back[:102]) + sum(t.fwd[:102]) + t.dropped_overrange
    oel, oaz = np.array(oel), np.array(oaz)
    for name, r, o in (("elevation", rel, oel), ("azimuth", raz, oaz)):
        p = compare_spectra(r.sum(0), 40000, o.sum(0), 20000)
        print("%s chi-squared p %.3g" % (name, p))
        assert p > 1e-3, (name, p)
