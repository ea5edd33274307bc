"""Whole runs of the CUDA engine against whole runs of the reference's own CPU code.

The reference runs (tests/golden/runs_*.txt.gz, written by tests/golden/make_runs.py) replay the
same scenes through the reference's classes: the PMMA linescan lines (config 2, the full 256 pixels
at 2000 primaries and 6 landing points in 16 batches), the rough-line layout (config 3's 385
regions), a feature scene with a cylinder, a rounded line and a block, the 10 keV deep layout
(config 5's features), NISTMottRS methods 2 and 3 on Si and PMMA, and Si with the phonon mechanism.

Trajectories draw different random numbers on each side, so the comparison is statistical:
  * yields: BSE and SE yields per landing point from independent batches on each side; z is the
    normal equivalent of the pooled t statistic of the difference of the means.  Each test is a
    family of k comparisons held to the false-alarm probability of one comparison at 3 standard
    errors (Sidak: |z| < 3.69 for k = 12), and the sum of all z^2 must pass a chi-squared test
    (p > 1e-3);
  * spectra: the back- and forward-scattered energy spectra of every landing point pass a
    two-sample chi-squared test, family-wise at 1e-3 (p > 1e-3 / k);
  * per-pixel image (the linescan): per-pixel BSE and SE z with each pixel's variance from the
    engine's 16 batches of that pixel (the t statistic with 15 degrees of freedom, converted to its
    normal equivalent); max |z| within the family bound for 512 comparisons, the sum of z^2 over the
    256 pixels chi-squared p > 1e-3 for each yield, and the scan's summed spectrum.
"""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

FP64, FP32 = 0, 1
OPT_EXACT_CSG = 2

sys.path.insert(0, GOLDEN)


def ref_set(name):
    import make_runs
    return make_runs.load(name)


def scene_of(name):
    from cudamonsel_b200 import scenes
    return {
        "lines_points": scenes.lines,
        "linescan": scenes.lines,
        "rough_points": lambda: scenes.rough_lines(seed=4),
        "features_ref_points": scenes.features_ref,
        "deep_points": lambda: scenes.deep_features(seed=3, cells=4, cell=320e-9)[0],
        "si_mott2": lambda: scenes.halfspace(mott_method=2),
        "si_mott3": lambda: scenes.halfspace(mott_method=3),
        "pmma_mott2": lambda: scenes.halfspace(material="pmma", mott_method=2),
        "pmma_mott3": lambda: scenes.halfspace(material="pmma", mott_method=3),
        "si_phonon": lambda: scenes.halfspace(phonon=True),
    }[name]()


def engine_batches(name, prec, batches=16, options=0, seed=1):
    """The reference set's landing points on the engine, `batches` batches of the reference's primaries per
    point.  Returns (back[batches, npts, bins], fwd[...], the reference set)."""
    from cudamonsel_b200 import capi, scenes
    ref = ref_set(name)
    e = capi.Engine(0)
    try:
        h = scenes.build_engine(scene_of(name), e)
        e.set_options(options)
        c = ref["centers"]
        cen = np.tile(c, (batches, 1))  # batch-major: rows b * npts + i
        back, fwd, st = e.run(h["chamber"], cen, scenes.eV(ref["beam_eV"]), ref["nprim"], ref["nbins"],
                              ref["width"], seed, precision=prec)
        assert st.primaries == len(cen) * ref["nprim"]
    finally:
        e.close()
    npts, nb = len(c), ref["nbins"] + 2
    return back.reshape(batches, npts, nb).astype(np.int64), fwd.reshape(batches, npts, nb).astype(np.int64), ref


def compare_points(eb, ef, ref, label):
    """Family-wise 3-sigma yields and 1e-3 spectra at every landing point; prints the z table."""
    from cudamonsel_b200 import scenes, stats
    rb, rf = ref["back"], ref["fwd"]
    beam, nbins, n_e, n_r = ref["beam_eV"], ref["nbins"], ref["nprim"], ref["nprim"]
    npts = rb.shape[1]
    zs = []
    worst_p = 1.0
    k = 2 * npts
    bound = stats.family_z_bound(k)
    for i in range(npts):
        ye = scenes.yields(eb[:, i], n_e, beam, nbins)
        yr = scenes.yields(rb[:, i], n_r, beam, nbins)
        row = []
        for j, nm in ((0, "BSE"), (1, "SE")):
            z, me, mr, se = stats.pooled_z(ye[j], yr[j])
            zs.append(z)
            row.append("%s %.4f/%.4f z=%+.2f" % (nm, me, mr, z))
        ps = []
        for name, he, hr in (("back", eb[:, i].sum(0), rb[:, i].sum(0)), ("fwd", ef[:, i].sum(0), rf[:, i].sum(0))):
            _, _, p = stats.chi2_two_sample(he, len(eb) * n_e, hr, len(rb) * n_r)
            ps.append(p)
        worst_p = min(worst_p, min(ps))
        x = ref["centers"][i]
        print("%s (%.0f, %.0f) nm  %s  spectra p %.3g %.3g" % (label, x[0] * 1e9, x[1] * 1e9, "  ".join(row), *ps))
    chi, dof, p = stats.chi2_of_z(zs)
    print("%s: max |z| %.2f (family bound %.2f for %d), sum z^2 %.1f / %d dof p %.3g, min spectrum p %.3g" % (
        label, np.max(np.abs(zs)), bound, k, chi, dof, p, worst_p))
    assert np.max(np.abs(zs)) < bound
    assert p > 1e-3
    assert worst_p > 1e-3 / (2 * npts)


POINT_SETS = ["lines_points", "rough_points", "features_ref_points", "deep_points", "si_mott2", "si_mott3",
              "pmma_mott2", "pmma_mott3", "si_phonon"]


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("name", POINT_SETS)
def test_points_match_reference(name, prec):
    """Yields and spectra at the set's landing points: engine 16 batches vs the reference's batches."""
    eb, ef, ref = engine_batches(name, prec, seed=11)
    compare_points(eb, ef, ref, "%s %s" % (name, "fp64" if prec == FP64 else "fp32"))


def test_lines_exact_csg_match_reference():
    """FP32 with the reference's NormalIntersectionShape march kept (CM_OPT_EXACT_CSG) instead of the
    merged plane sets."""
    eb, ef, ref = engine_batches("lines_points", FP32, options=OPT_EXACT_CSG, seed=12)
    compare_points(eb, ef, ref, "lines_points fp32 exact-csg")


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_linescan_image_matches_reference(prec):
    """The full config-2 linescan (256 pixels, 1 nm apart, 2000 primaries each): per-pixel BSE and SE
    yields of the engine (16 batches of 2000 per pixel) against the reference's single run per pixel."""
    from cudamonsel_b200 import scenes, stats
    eb, ef, ref = engine_batches("linescan", prec, seed=13)
    beam, nbins, n = ref["beam_eV"], ref["nbins"], ref["nprim"]
    B, npix = eb.shape[0], eb.shape[1]
    ye = [np.zeros((B, npix)), np.zeros((B, npix))]
    for b in range(B):
        y = scenes.yields(eb[b], n, beam, nbins)
        ye[0][b], ye[1][b] = y
    yr = scenes.yields(ref["back"][0], n, beam, nbins)
    bound = stats.family_z_bound(2 * npix)
    zall = []
    for j, nm in ((0, "BSE"), (1, "SE")):
        me = ye[j].mean(0)
        z = stats.scan_z(ye[j], n, yr[j], n)
        chi, dof, p = stats.chi2_of_z(z)
        zall.append(z)
        worst = int(np.argmax(np.abs(z)))
        print("%s per pixel: mean engine %.4f ref %.4f; max |z| %.2f at x = %.1f nm; |z| > 3 at %d of %d; "
              "rms z %.3f; sum z^2 %.1f / %d p %.3g" % (nm, me.mean(), yr[j].mean(), abs(z[worst]),
                                                      ref["centers"][worst][0] * 1e9, int((np.abs(z) > 3).sum()),
                                                      npix, np.sqrt((z * z).mean()), chi, dof, p))
        assert p > 1e-3
    assert np.max(np.abs(np.concatenate(zall))) < bound
    _, dof, p = stats.chi2_two_sample(eb.sum((0, 1)), B * npix * n, ref["back"].sum((0, 1)), npix * n)
    print("scan spectrum chi2 p %.3g (%d dof)" % (p, dof))
    assert p > 1e-3
