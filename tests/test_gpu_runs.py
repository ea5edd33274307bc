"""Whole-run parity of the CUDA engine with the reference and the oracle.

Trajectories use different random streams on each side, so the comparison is
statistical: yields per batch (a batch = one pixel of N primaries at the same
landing point) give the standard errors; the BSE and SE yields of all landing
points of a test must agree within 3 standard errors family-wise (Sidak over
the test's comparisons), the sum of their z^2 must pass a chi-squared test
(p > 1e-3), and the back-scattered energy spectra must pass a two-sample
chi-squared test (p > 1e-3, family-wise).  FP32 must also sit within 1 % of FP64.
Runs against the reference's own whole runs are in test_gpu_reference_runs.py.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

FP64, FP32 = 0, 1


def ref_runs():
    runs = []
    for line in open(os.path.join(GOLDEN, "run_halfspace_1keV.txt")):
        w = line.split()
        if w and w[0] == "back":
            runs.append([int(x) for x in w[1:]])
    return np.array(runs)


def batch_yields(back, nprim, beam_eV, nbins):
    from cudamonsel_b200 import scenes
    return scenes.yields(back, nprim, beam_eV, nbins)


@pytest.fixture(scope="module")
def half(engine):
    from cudamonsel_b200 import scenes
    sc = scenes.halfspace()
    return engine, scenes.build_engine(sc, engine)


def run_half(engine, h, prec, npix, nprim, seed, energy_eV=1000.0):
    from cudamonsel_b200 import scenes
    centers = np.tile([0.0, 0.0, -20e-9], (npix, 1))
    nb = int(energy_eV / 10)
    back, fwd, st = engine.run(h["chamber"], centers, scenes.eV(energy_eV), nprim, nb, 0.0, seed, precision=prec)
    return back, fwd, st


def test_halfspace_fp64_matches_reference(half):
    """1 keV pencil beam on flat Si (the reference's configs[0] path): engine FP64, 40 x 1000
    primaries, vs the reference's 4 x 10 000."""
    from cudamonsel_b200 import stats
    e, h = half
    back, fwd, st = run_half(e, h, FP64, 40, 1000, seed=5)
    assert st.primaries == 40000
    bse, se = batch_yields(back, 1000, 1000.0, 100)
    ref = ref_runs()
    rb, rs = batch_yields(ref, 10000, 1000.0, 100)
    # reference batches are 10x larger: scale their spread to the engine's batch size
    zb = (bse.mean() - rb.mean()) / np.sqrt(bse.var(ddof=1) / len(bse) * (1 + len(bse) / (len(rb) * 10)))
    zs = (se.mean() - rs.mean()) / np.sqrt(se.var(ddof=1) / len(se) * (1 + len(se) / (len(rs) * 10)))
    print("BSE engine %.4f ref %.4f z=%.2f | SE engine %.4f ref %.4f z=%.2f" % (bse.mean(), rb.mean(), zb, se.mean(),
                                                                              rs.mean(), zs))
    assert abs(zb) < 3 and abs(zs) < 3
    chi, dof, p = stats.chi2_two_sample(back.sum(0), 40000, ref.sum(0), 40000)
    print("spectrum chi2 %.1f dof %d p %.3g" % (chi, dof, p))
    assert p > 1e-3


def test_halfspace_fp32_within_1pct_of_fp64(half):
    """FP32 transport (FP64 positions and plane solves) vs FP64 on 200 x 2000 primaries each."""
    from cudamonsel_b200 import stats
    e, h = half
    b64, _, _ = run_half(e, h, FP64, 200, 2000, seed=11)
    b32, _, _ = run_half(e, h, FP32, 200, 2000, seed=12)
    y64 = batch_yields(b64, 2000, 1000.0, 100)
    y32 = batch_yields(b32, 2000, 1000.0, 100)
    for name, a, b in (("BSE", y32[0], y64[0]), ("SE", y32[1], y64[1])):
        z = stats.z_score(a, b)
        relerr = abs(a.mean() - b.mean()) / b.mean()
        print("%s fp32 %.5f fp64 %.5f rel %.4f z %.2f" % (name, a.mean(), b.mean(), relerr, z))
        assert abs(z) < 3
        assert relerr < 0.01
    chi, dof, p = stats.chi2_two_sample(b32.sum(0), 400000, b64.sum(0), 400000)
    print("spectrum chi2 %.1f dof %d p %.3g" % (chi, dof, p))
    assert p > 1e-3


def oracle_points(sc, centers, width, energy, nprim, seed, nbins, batches=4):
    """The oracle's whole trajectories at each landing point in `batches` batches of nprim:
    back[batches, npts, nbins + 2]."""
    import pyoracle
    ob, of, tl = pyoracle.run_scene(sc, np.tile(centers, (batches, 1)), width, energy, nprim, seed, nbins)
    return ob.reshape(batches, len(centers), nbins + 2)


def assert_points_agree(eng_back, n_e, ora_back, n_o, beam_eV, nbins, label, xs):
    """Engine batches against oracle batches at each landing point: pooled-t z of BSE and SE yields held
    family-wise to 3 standard errors (Sidak over the 2 x points comparisons), sum of z^2 chi-squared
    p > 1e-3, and each point's back-scattered spectrum p > 1e-3 / points."""
    from cudamonsel_b200 import stats
    npts = ora_back.shape[1]
    zs, ps = [], []
    for i in range(npts):
        ye = batch_yields(eng_back[:, i], n_e, beam_eV, nbins)
        yo = batch_yields(ora_back[:, i], n_o, beam_eV, nbins)
        row = []
        for j, nm in ((0, "BSE"), (1, "SE")):
            z, me, mo, _ = stats.pooled_z_weighted(ye[j], n_e, yo[j], n_o)
            zs.append(z)
            row.append("%s %.4f/%.4f z=%+.2f" % (nm, me, mo, z))
        p = stats.chi2_two_sample(eng_back[:, i].sum(0), len(eng_back) * n_e, ora_back[:, i].sum(0),
                                  len(ora_back) * n_o)[2]
        ps.append(p)
        print("%s x=%6.1f nm  %s  spectrum p %.3g" % (label, xs[i] * 1e9, "  ".join(row), p))
    chi, dof, p = stats.chi2_of_z(zs)
    bound = stats.family_z_bound(len(zs))
    print("%s: max |z| %.2f (bound %.2f), sum z^2 %.1f / %d p %.3g" % (label, np.max(np.abs(zs)), bound, chi, dof, p))
    assert np.max(np.abs(zs)) < bound
    assert p > 1e-3
    assert min(ps) > 1e-3 / npts


def engine_points(e, chamber, centers, energy, nprim, nbins, width, seed, prec, batches=16):
    """Engine batches at each landing point: back[batches, npts, nbins + 2]."""
    back, fwd, st = e.run(chamber, np.tile(centers, (batches, 1)), energy, nprim, nbins, width, seed=seed,
                          precision=prec)
    return back.reshape(batches, len(centers), nbins + 2).astype(np.int64)


LINE_XS = np.array([-60.0, -22.0, -19.0, -12.0, 0.0, 100.0]) * 1e-9


@pytest.fixture(scope="module")
def lines_oracle_runs():
    from cudamonsel_b200 import scenes
    centers = np.stack([LINE_XS, np.zeros(6), np.full(6, -120e-9)], axis=1)
    return centers, oracle_points(scenes.lines(), centers, 1e-9, scenes.eV(500.0), 500, 77, 50)


@pytest.mark.parametrize("prec,options", [(FP64, 0), (FP32, 0), (FP32, 2)], ids=["fp64", "fp32", "fp32-exact-csg"])
def test_lines_match_oracle(lines_oracle_runs, prec, options):
    """PMMA lines on Si, 500 eV, sigma 1 nm: 6 landing points (gap, sidewall foot, sidewall,
    top), engine vs the oracle's whole trajectories.  FP32 runs with the lines merged into
    single plane sets (default) and with the reference's intersection march (CM_OPT_EXACT_CSG,
    set after the scene is built: building a scene applies the scene's own options)."""
    from cudamonsel_b200 import capi, scenes
    centers, ob = lines_oracle_runs
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.lines(), e)
    e.set_options(options)
    back = engine_points(e, h["chamber"], centers, scenes.eV(500.0), 500, 50, 1e-9, 3, prec)
    e.close()
    assert_points_agree(back, 500, ob, 500, 500.0, 50, "lines", LINE_XS)


FEATURE_XS = np.array([-60.0, -35.0, 40.0, 60.0, 82.0]) * 1e-9


@pytest.fixture(scope="module")
def features_oracle_runs():
    from cudamonsel_b200 import scenes
    centers = np.stack([FEATURE_XS, np.zeros(5), np.full(5, -120e-9)], axis=1)
    return centers, oracle_points(scenes.features(), centers, 1e-9, scenes.eV(800.0), 500, 91, 80)


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_features_match_oracle(features_oracle_runs, prec):
    """NormalCylindricalShape, the rounded createLine (NormalUnionShape of plane sets and cylinders)
    and a block on Si at 800 eV with the JMONSEL fixes on (refraction, the d3 abscissae, the left
    rounded corner): engine vs the oracle's whole trajectories at 5 landing points."""
    from cudamonsel_b200 import capi, scenes
    centers, ob = features_oracle_runs
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.features(), e)
    back = engine_points(e, h["chamber"], centers, scenes.eV(800.0), 500, 80, 1e-9, 5, prec)
    e.close()
    assert_points_agree(back, 500, ob, 500, 800.0, 80, "features", FEATURE_XS)


ROUGH_XS = np.array([-219.0, -200.0, -180.0, -21.0, 1.0, 21.0]) * 1e-9


@pytest.fixture(scope="module")
def rough_oracle_runs():
    from cudamonsel_b200 import scenes
    centers = np.stack([ROUGH_XS, np.linspace(-40e-9, 40e-9, 6), np.full(6, -120e-9)], axis=1)
    return centers, oracle_points(scenes.rough_lines(seed=4), centers, 1e-9, scenes.eV(500.0), 500, 13, 50)


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_rough_lines_match_oracle(rough_oracle_runs, prec):
    """The rough-line layout (3 lines x 128 segments with N(0, 1.5 nm) sidewall offsets, 385 regions
    under the chamber) at 500 eV: engine vs oracle at 6 landing points on and beside the edges."""
    from cudamonsel_b200 import capi, scenes
    centers, ob = rough_oracle_runs
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.rough_lines(seed=4), e)
    back = engine_points(e, h["chamber"], centers, scenes.eV(500.0), 500, 50, 1e-9, 21, prec)
    e.close()
    assert_points_agree(back, 500, ob, 500, 500.0, 50, "rough", ROUGH_XS)


@pytest.fixture(scope="module")
def mott_method_oracle_runs():
    from cudamonsel_b200 import scenes
    out = {}
    for mat in ("si", "pmma"):
        for method in (2, 3):
            sc = scenes.halfspace(material=mat, mott_method=method)
            out[mat, method] = oracle_points(sc, np.array([[0.0, 0.0, -20e-9]]), 0.0, scenes.eV(300.0), 2000, 31,
                                             30, batches=8)
    return out


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("method", [2, 3])
@pytest.mark.parametrize("mat", ["si", "pmma"])
def test_nistmott_methods_match_oracle(mott_method_oracle_runs, mat, method, prec):
    """Flat Si and PMMA at 300 eV with NISTMottRS method 2 (Factory100) or 3 (Factory100Lin): most of the
    secondaries scatter elastically below 100 eV, where the methods differ (method 3 raises the SE yield by
    a quarter), so the yields test the per-mechanism method choice.  Engine 64 x 500 primaries vs the
    oracle's 8 x 2000; the same seed with method 1 must give different tallies."""
    from cudamonsel_b200 import capi, scenes
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.halfspace(material=mat, mott_method=method), e)
    centers = np.array([[0.0, 0.0, -20e-9]])
    back = engine_points(e, h["chamber"], centers, scenes.eV(300.0), 500, 30, 0.0, 41, prec, batches=64)
    e.reset()
    h1 = scenes.build_engine(scenes.halfspace(material=mat, mott_method=1), e)
    back1 = engine_points(e, h1["chamber"], centers, scenes.eV(300.0), 500, 30, 0.0, 41, prec, batches=64)
    e.close()
    assert not np.array_equal(back, back1)
    assert_points_agree(back, 500, mott_method_oracle_runs[mat, method], 2000, 300.0, 30,
                        "%s method %d" % (mat, method), [0.0])


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_child_grid_finds_what_the_scan_finds(prec):
    """The rough-line chamber (385 children) searched through its x-y grid and by the in-order scan
    (CM_OPT_SCAN_CHILDREN) gives identical tallies on a 24 x 24 image at 300-1000 eV."""
    from cudamonsel_b200 import capi, scenes
    ic, ie, inp, inb = scenes.rough_image(seed=2, side=24, mean_nprim=150)
    keys = np.arange(len(ic), dtype=np.uint64) + np.uint64(99)
    out = []
    for opt in (0, 4):
        e = capi.Engine(0)
        sc = scenes.rough_lines(seed=2)
        sc.spec.options = opt
        h = scenes.build_engine(sc, e)
        back, fwd, st = e.run(h["chamber"], ic, ie, inp, inb, 1e-9, 0, precision=prec, pixel_keys=keys)
        e.close()
        out.append((back, fwd, st.steps))
    assert out[0][2] == out[1][2]
    assert (out[0][0] == out[1][0]).all() and (out[0][1] == out[1][1]).all()


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_deep_features_match_oracle(prec):
    """4 x 4 seed-placed blocks and cylinders on Si at 10 keV: engine vs oracle at 4 landing points."""
    from cudamonsel_b200 import capi, scenes
    sc, top = scenes.deep_features(seed=3, cells=4, cell=320e-9)
    xs = np.array([-480.0, -160.0, 160.0, 480.0]) * 1e-9
    centers = np.stack([xs, np.array([-160.0, 160.0, -160.0, 160.0]) * 1e-9, np.full(4, -(top + 20e-9))], axis=1)
    ob = oracle_points(sc, centers, 1e-9, scenes.eV(10000.0), 100, 17, 1000)
    e = capi.Engine(0)
    h = scenes.build_engine(sc, e)
    back = engine_points(e, h["chamber"], centers, scenes.eV(10000.0), 100, 1000, 1e-9, 23, prec)
    e.close()
    assert_points_agree(back, 100, ob, 100, 10000.0, 1000, "deep", xs)


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_tail_steps_give_the_same_tallies(prec):
    """The tail of a run (fewer electrons left than fill the GPU) runs several whole steps per thread
    (k_steps); CM_OPT_QUEUE_STEPS keeps the queue kernels to the end, and a profiled run times each
    kernel.  Same seed: identical tallies all three ways."""
    from cudamonsel_b200 import capi, scenes
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.lines(), e)
    c = scenes.linescan_pixels(64)
    b0, f0, s0 = e.run(h["chamber"], c, scenes.eV(500.0), 300, 50, 1e-9, seed=9, precision=prec)
    b2, f2, s2 = e.run(h["chamber"], c, scenes.eV(500.0), 300, 50, 1e-9, seed=9, precision=prec, profile=1)
    e.set_options(capi.OPT_QUEUE_STEPS)
    b1, f1, s1 = e.run(h["chamber"], c, scenes.eV(500.0), 300, 50, 1e-9, seed=9, precision=prec)
    e.close()
    print("steps %d, tail launches %d of %d iterations, %d electrons started in k_steps" % (
        s0.steps, s0.step_launches, s0.iterations, s0.step_units))
    assert s0.step_launches > 0 and s1.step_launches == 0 and s2.step_launches > 0
    assert s2.step_ms > 0 and s2.kernel_ms[0] > 0 and s1.step_units == 0
    for b, f, s in ((b1, f1, s1), (b2, f2, s2)):
        assert s0.steps == s.steps and s0.secondaries == s.secondaries
        assert np.array_equal(b0, b) and np.array_equal(f0, f)


def ref_angles(kind):
    runs = []
    for line in open(os.path.join(GOLDEN, "run_halfspace_1keV.txt")):
        w = line.split()
        if w and w[0] == kind:
            runs.append([int(x) for x in w[1:]])
    return np.array(runs)


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_angle_histograms_match_reference(half, prec):
    """BackscatterStats' elevation and azimuthal histograms (BackscatterStats.cu:105-106,147-165), 1 keV
    pencil beam on flat Si: engine 40 x 1000 primaries vs the reference's 4 x 10 000 (chi-squared)."""
    from cudamonsel_b200 import stats
    e, h = half
    centers = np.tile([0.0, 0.0, -20e-9], (40, 1))
    back, fwd, st, ex = e.run(h["chamber"], centers, scenes_eV(1000.0), 1000, 100, 0.0, seed=21, precision=prec,
                              angles=True)
    el, az = ex["elevation"], ex["azimuth"]
    assert el.shape == (40, 182) and az.shape == (40, 362)
    assert el.sum() == az.sum() == st.escapes
    assert el.sum() >= back.sum() + fwd.sum() and el[:, :92].sum() == 0
    for name, mine in (("elev", el), ("azim", az)):
        ref = ref_angles(name)
        chi, dof, p = stats.chi2_two_sample(mine.sum(0), 40000, ref.sum(0), 40000)
        print("%s chi2 %.1f dof %d p %.3g" % (name, chi, dof, p))
        assert p > 1e-3


def scenes_eV(x):
    from cudamonsel_b200 import scenes
    return scenes.eV(x)


def ref_bin(maxv, nbins, vals):
    """Histogram(0, max, nbins).bin + 1 with Algorithm::binarySearch's insertion point (the tallies' rule)."""
    delta = maxv / nbins
    edges = np.array([0.0] + [0.0 + i * delta for i in range(1, nbins + 1)])
    return np.searchsorted(edges, vals, side="left") + 1


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_escape_log_rebuilds_the_tallies(prec):
    """BackscatterStats' detected-electron log: one record per escape; binning the logged energies and
    escape points again gives the run's energy histograms exactly and its angle histograms up to the
    rounding of the logged position; a smaller log keeps the first records and the count."""
    from cudamonsel_b200 import capi, scenes
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.lines(), e)
    c = scenes.linescan_pixels(16)
    back, fwd, st, ex = e.run(h["chamber"], c, scenes.eV(500.0), 200, 50, 1e-9, seed=4, precision=prec, angles=True,
                              escape_log_cap=200000)
    log = ex["escape_log"]
    assert len(log) == st.escapes > 0
    assert len(np.unique(log["pixel"])) == 16 and (log["step"] > 0).all()
    pos = log["position"]
    elev = np.pi / 2 - np.arctan2(pos[:, 2], np.sqrt(pos[:, 0] ** 2 + pos[:, 1] ** 2))
    e0ref = scenes.eV(500.0) * (1.0 / 1.60217653e-19)  # the histogram top as the engine computes it (FromSI::eV)
    be = ref_bin(e0ref, 50, log["energy_eV"])
    for px in range(16):
        m = log["pixel"] == px
        for hist, sel in ((back, elev[m] >= np.pi / 2), (fwd, elev[m] < np.pi / 2)):
            b = be[m][sel]
            counts = np.bincount(b[b <= 51], minlength=52)
            assert np.array_equal(counts, hist[px].astype(np.int64)), px
    el_counts = np.bincount(ref_bin(np.pi, 180, elev), minlength=182)
    diff = np.abs(el_counts - ex["elevation"].sum(0).astype(np.int64)).sum()
    print("escapes %d, elevation histogram from the log differs by %d counts" % (st.escapes, diff))
    assert diff <= 4
    d = np.stack([np.cos(log["phi"]) * np.sin(log["theta"]), np.sin(log["phi"]) * np.sin(log["theta"]),
                  np.cos(log["theta"])], axis=1)
    assert np.allclose((d * d).sum(1), 1.0)
    _, _, st2, ex2 = e.run(h["chamber"], c, scenes.eV(500.0), 200, 50, 1e-9, seed=4, precision=prec,
                           escape_log_cap=100)
    e.close()
    assert st2.escapes == st.escapes and len(ex2["escape_log"]) == 100


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_angle_histograms_and_log_through_run_device(prec):
    """cm_run_device with device arrays for the angle histograms and the escape log (filled with garbage
    first: the run clears the histograms) gives what cm_run gives with host arrays for the same keys."""
    import ctypes as C
    import torch
    from cudamonsel_b200 import capi, scenes
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.lines(), e)
    npix, nprim, nb = 24, 150, 50
    c = scenes.linescan_pixels(npix)
    keys = np.arange(npix, dtype=np.uint64) + np.uint64(777)
    back, fwd, st, ex = e.run(h["chamber"], c, scenes.eV(500.0), nprim, nb, 1e-9, 0, precision=prec, angles=True,
                              escape_log_cap=100000, pixel_keys=keys)
    dev = torch.device("cuda", 0)
    tc = torch.tensor(c.ravel(), dtype=torch.float64, device=dev)
    te = torch.full((npix,), scenes.eV(500.0), dtype=torch.float64, device=dev)
    tn = torch.full((npix,), nprim, dtype=torch.int32, device=dev)
    tb = torch.full((npix,), nb, dtype=torch.int32, device=dev)
    tk = torch.tensor(keys.astype(np.int64), device=dev)
    tback = torch.zeros((npix, nb + 2), dtype=torch.int32, device=dev)
    tfwd = torch.zeros_like(tback)
    tel = torch.full((npix, capi.ELEVATION_COUNTS), 9, dtype=torch.int32, device=dev)
    taz = torch.full((npix, capi.AZIMUTH_COUNTS), 9, dtype=torch.int32, device=dev)
    tlog = torch.zeros((100000, capi.ESCAPE_RECORD.itemsize // 8), dtype=torch.int64, device=dev)
    P = lambda x, ty: C.cast(C.c_void_p(x.data_ptr()), C.POINTER(ty))
    d = capi.RunDesc(h["chamber"], prec, npix, 1e-9, P(tc, C.c_double), P(te, C.c_double), P(tn, C.c_int),
                     P(tb, C.c_int), 0, nb + 2, 0, 0, P(tk, C.c_uint64), 0)
    d.elevation = P(tel, C.c_uint32)
    d.azimuth = P(taz, C.c_uint32)
    d.escape_log = tlog.data_ptr()
    d.escape_log_cap = 100000
    st2 = e.run_device(d, tback.data_ptr(), tfwd.data_ptr())
    torch.cuda.synchronize()
    e.close()
    assert st2.escapes == st.escapes
    assert np.array_equal(tback.cpu().numpy().astype(np.uint32), back)
    assert np.array_equal(tel.cpu().numpy().astype(np.uint32), ex["elevation"])
    assert np.array_equal(taz.cpu().numpy().astype(np.uint32), ex["azimuth"])
    log2 = tlog.cpu().numpy()[:st2.escapes].copy().view(capi.ESCAPE_RECORD).ravel()
    order = lambda g: np.lexsort((g["step"], g["electron"]))
    a, b = ex["escape_log"][order(ex["escape_log"])], log2[order(log2)]
    assert np.array_equal(a["electron"], b["electron"]) and np.array_equal(a["energy_eV"], b["energy_eV"])


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_autotune_and_settings_keep_the_tallies(prec):
    """cm_autotune keeps the fastest launch settings for the precision it tuned; runs under the tuned,
    the default and deliberately odd settings (small waves, short tail steps, few blocks) give the
    same tallies.  Out-of-range settings are refused."""
    from cudamonsel_b200 import capi, scenes
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.lines(), e)
    c = scenes.linescan_pixels(32)
    args = (h["chamber"], c, scenes.eV(500.0), 300, 50, 1e-9, 9)
    with pytest.raises(capi.CMError):
        e.set_tuning(prec, blocks_per_sm=64)
    b0, f0, s0 = e.run(*args, precision=prec)
    t = e.autotune(*args, precision=prec)
    print("tuned", t.as_dict())
    got = e.tuning(prec)
    assert t.ms > 0 and (got.wave, got.tail_below, got.tail_steps, got.blocks_per_sm) == (
        t.wave, t.tail_below, t.tail_steps, t.blocks_per_sm)
    other = e.tuning(FP32 if prec == FP64 else FP64)
    assert (other.wave, other.tail_below, other.tail_steps, other.blocks_per_sm) == (0, 0, 0, 0)
    b1, f1, s1 = e.run(*args, precision=prec)
    e.set_tuning(prec, wave=65536, tail_below=3000, tail_steps=3, blocks_per_sm=2)
    b2, f2, s2 = e.run(*args, precision=prec)
    e.close()
    for b, f, s in ((b1, f1, s1), (b2, f2, s2)):
        assert s.steps == s0.steps and np.array_equal(b, b0) and np.array_equal(f, f0)


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_staged_tables_give_the_same_tallies(prec):
    """The event kernels read the small tables from shared memory (a bulk copy per block);
    CM_OPT_GLOBAL_TABLES reads them from global memory.  Same seed: identical tallies, for the lines
    (Si and PMMA tables) and for a run whose tail goes to k_steps."""
    from cudamonsel_b200 import capi, scenes
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.lines(), e)
    c = scenes.linescan_pixels(48)
    b0, f0, s0 = e.run(h["chamber"], c, scenes.eV(500.0), 300, 50, 1e-9, seed=12, precision=prec)
    e.set_options(capi.OPT_GLOBAL_TABLES)
    b1, f1, s1 = e.run(h["chamber"], c, scenes.eV(500.0), 300, 50, 1e-9, seed=12, precision=prec)
    e.close()
    assert s0.step_launches > 0
    assert s0.steps == s1.steps and np.array_equal(b0, b1) and np.array_equal(f0, f1)


@pytest.fixture(scope="module")
def penn_runs(tmp_path_factory):
    """Scattering tables from the dielectric model (small grids) and oracle runs on them."""
    import pyoracle
    from cudamonsel_b200 import scenes
    from cudamonsel_b200.data import gen_penn_tables, gen_si_tables
    d = str(tmp_path_factory.mktemp("penn"))
    gen_penn_tables.build(d, n_iimfp=48, n_loss=24, n_theta=(16, 17, 17))
    tables = [os.path.join(d, n) for n in gen_si_tables.NAMES]
    ob, _, _ = pyoracle.run_scene(scenes.halfspace(tables=tables), np.tile([0.0, 0.0, -20e-9], (8, 1)), 0.0,
                                  scenes.eV(1000.0), 1500, 51, 100)
    return tables, ob


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_penn_tables_match_oracle(penn_runs, prec):
    """Tables generated from the dielectric model (Penn single-pole algorithm) run on the engine: flat Si,
    1 keV, engine 32 x 500 primaries vs the oracle's 8 x 1500 on the same tables."""
    from cudamonsel_b200 import capi, scenes, stats
    tables, ob = penn_runs
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.halfspace(tables=tables), e)
    back, _, st = e.run(h["chamber"], np.tile([0.0, 0.0, -20e-9], (32, 1)), scenes.eV(1000.0), 500, 100, 0.0,
                        seed=8, precision=prec)
    e.close()
    assert_points_agree(back.reshape(32, 1, -1).astype(np.int64), 500, ob.reshape(8, 1, -1), 1500, 1000.0, 100,
                        "penn tables", [0.0])


def test_deterministic_and_independent_of_batch(half):
    """Same seed -> identical tallies; a pixel's tally is the same alone and inside a larger
    batch of other pixels when it carries the same stream key (the serving guarantee)."""
    from cudamonsel_b200 import scenes
    e, h = half
    c = np.array([[0.0, 0.0, -20e-9]])
    k = np.array([12345], dtype=np.uint64)
    a, _, _ = e.run(h["chamber"], c, scenes.eV(1000.0), 300, 100, 0.0, 1, precision=FP64, pixel_keys=k)
    b, _, _ = e.run(h["chamber"], c, scenes.eV(1000.0), 300, 100, 0.0, 1, precision=FP64, pixel_keys=k)
    assert (a == b).all()
    many = np.tile(c, (50, 1))
    keys = np.arange(1000, 1050, dtype=np.uint64)
    keys[17] = 12345
    m, _, _ = e.run(h["chamber"], many, scenes.eV(1000.0), 300, 100, 0.0, 9, precision=FP64, pixel_keys=keys)
    assert (m[17] == a[0]).all()
    assert not (m[16] == a[0]).all()
    a32, _, _ = e.run(h["chamber"], c, scenes.eV(1000.0), 300, 100, 0.0, 1, precision=FP32, pixel_keys=k)
    m32, _, _ = e.run(h["chamber"], many, scenes.eV(1000.0), 300, 100, 0.0, 9, precision=FP32, pixel_keys=keys)
    assert (m32[17] == a32[0]).all()


def test_edge_cases(half):
    """Empty pixels, a single primary, nbins at both ends, energies below the tracking cut."""
    from cudamonsel_b200 import scenes
    e, h = half
    c = np.tile([0.0, 0.0, -20e-9], (4, 1))
    back, fwd, st = e.run(h["chamber"], c, scenes.eV(1000.0), [0, 1, 0, 5], [1, 100, 1024, 7], 0.0, 2)
    assert back.shape == (4, 1026)
    assert back[0].sum() == 0 and back[2].sum() == 0
    assert st.primaries == 6
    # a 2 eV beam: below Si's 3.75 eV barrier after entering? (it gains 3.75 eV entering) -> tracked
    back, fwd, st = e.run(h["chamber"], c[:1], scenes.eV(2.0), 50, 1, 0.0, 3)
    assert st.primaries == 50


def test_oversized_wave_is_enomem_and_the_context_stays_usable(half):
    """A wave whose run buffers exceed the device's free memory (2^27 electrons in FP64: about 240 GB) is
    refused with CM_ENOMEM before anything is allocated; a wave beyond 2^27 is CM_EINVAL; a normal run on
    the same context follows (the autotuner skips such a candidate the same way)."""
    from cudamonsel_b200 import capi, scenes
    e, h = half
    c = np.array([[0.0, 0.0, -20e-9]])
    with pytest.raises(capi.CMError, match="GB of run buffers") as ei:
        e.run(h["chamber"], c, scenes.eV(1000.0), 10, 100, 0.0, 1, precision=FP64, wave=1 << 27)
    assert ei.value.code == capi.ENOMEM
    with pytest.raises(capi.CMError) as ei:
        e.run(h["chamber"], c, scenes.eV(1000.0), 10, 100, 0.0, 1, precision=FP64, wave=(1 << 27) + 1)
    assert ei.value.code == capi.EINVAL
    back, fwd, st = e.run(h["chamber"], c, scenes.eV(1000.0), 10, 100, 0.0, 1, precision=FP64)
    assert st.primaries == 10 and back.sum() > 0


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_pool_overflow_restart_gives_the_same_tallies(prec):
    """A secondary pool of one record per wave electron (cm_tuning.pool = 1, wave 1024) overflows on 5 keV
    primaries; the run is repeated with twice the pool until it fits (pool_restarts > 0), and its tallies and
    counts are those of a run with the default pool, because every electron's stream is keyed by its lineage.
    The job server restarts a batch the same way."""
    from cudamonsel_b200 import capi, scenes
    c = np.tile([0.0, 0.0, -20e-9], (4, 1))
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.halfspace(), e)
    ref = e.run(h["chamber"], c, scenes.eV(5000.0), 100, 500, 0.0, 5, precision=prec)
    assert ref[2].pool_restarts == 0
    e.set_tuning(prec, wave=1024, pool=1)
    small = e.run(h["chamber"], c, scenes.eV(5000.0), 100, 500, 0.0, 5, precision=prec)
    assert small[2].pool_restarts > 0
    assert (small[0] == ref[0]).all() and (small[1] == ref[1]).all()
    assert small[2].steps == ref[2].steps and small[2].secondaries == ref[2].secondaries
    srv = capi.Server(0, slots=4, budget_gb=4.0)
    srv.tune(prec, wave=1024, pool=1)
    job = srv.submit(e, h["chamber"], c, scenes.eV(5000.0), 100, 500, 0.0, 5, precision=prec)
    assert srv.wait(job).state == capi.JOB_DONE
    b, f, st = srv.result(job)
    srv.close()
    e.close()
    assert st.pool_restarts > 0 and st.steps == ref[2].steps
    assert (b == ref[0]).all() and (f == ref[1]).all()


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_device_loop_limit_and_graph_reuse(half, prec):
    """The device-driven loop (one launch per run of a graph cached in the context): an iteration limit stops
    the run on the device with CM_ELIMIT; the following runs reuse the cached graph and give identical
    tallies and counts run after run, equal to a fresh context's and to a profiled run's (the host replays
    iterations there)."""
    from cudamonsel_b200 import capi, scenes
    e, h = half
    c = np.tile([0.0, 0.0, -20e-9], (16, 1))
    with pytest.raises(capi.CMError, match="iteration limit") as ei:
        e.run(h["chamber"], c, scenes.eV(1000.0), 200, 100, 0.0, 3, precision=prec, max_iterations=16)
    assert ei.value.code == capi.ELIMIT
    runs = [e.run(h["chamber"], c, scenes.eV(1000.0), 200, 100, 0.0, 3, precision=prec) for _ in range(3)]
    runs.append(e.run(h["chamber"], c, scenes.eV(1000.0), 200, 100, 0.0, 3, precision=prec, profile=1))
    fresh = capi.Engine(0)
    hf = scenes.build_engine(scenes.halfspace(), fresh)
    runs.append(fresh.run(hf["chamber"], c, scenes.eV(1000.0), 200, 100, 0.0, 3, precision=prec))
    fresh.close()
    b0, f0, s0 = runs[0]
    print("iterations %d, queue launches %d, tail launches %d; device ms %s" % (
        s0.iterations, s0.kernel_launches[0], s0.step_launches, [round(r[2].device_ms, 2) for r in runs]))
    assert s0.primaries == 16 * 200
    for k, (b, f, s) in enumerate(runs[1:], start=1):
        assert np.array_equal(b, b0) and np.array_equal(f, f0)
        assert s.steps == s0.steps and s.secondaries == s0.secondaries
        if k != 3:  # the profiled run switches to the tail at a replay boundary: other iteration counts
            assert s.iterations == s0.iterations
