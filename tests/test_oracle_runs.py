"""The oracle's whole runs against the reference's own whole runs (CPU, no GPU).

The oracle restates the reference's transport step by step (tests/test_oracle_golden.py pins every
function bit for bit); these tests pin whole trajectories on multi-region scenes as well, with the
same statistics the GPU tests use (tests/test_gpu_reference_runs.py): pooled-t yields per landing
point held family-wise to 3 standard errors, sum of z^2 chi-squared p > 1e-3, spectra p > 1e-3 / k.
"""
import sys

import numpy as np
import pytest

from conftest import GOLDEN

sys.path.insert(0, GOLDEN)


def oracle_batches(name, scene, batches, nprim, seed):
    import make_runs
    import pyoracle
    from cudamonsel_b200 import scenes
    ref = make_runs.load(name)
    c = ref["centers"]
    cen = np.tile(c, (batches, 1))
    ob, of, _ = pyoracle.run_scene(scene, cen, ref["width"], scenes.eV(ref["beam_eV"]), nprim, seed, ref["nbins"])
    nb = ref["nbins"] + 2
    return ob.reshape(batches, len(c), nb), of.reshape(batches, len(c), nb), ref


def check(ob, of, ref, nprim, label):
    from cudamonsel_b200 import scenes, stats
    npts = ref["back"].shape[1]
    zs, ps = [], []
    for i in range(npts):
        yo = scenes.yields(ob[:, i], nprim, ref["beam_eV"], ref["nbins"])
        yr = scenes.yields(ref["back"][:, i], ref["nprim"], ref["beam_eV"], ref["nbins"])
        for j in (0, 1):
            z, mo, mr, _ = stats.pooled_z_weighted(yo[j], nprim, yr[j], ref["nprim"])
            zs.append(z)
        for he, hr in ((ob[:, i].sum(0), ref["back"][:, i].sum(0)), (of[:, i].sum(0), ref["fwd"][:, i].sum(0))):
            ps.append(stats.chi2_two_sample(he, len(ob) * nprim, hr, len(ref["back"]) * ref["nprim"])[2])
    chi, dof, p = stats.chi2_of_z(zs)
    bound = stats.family_z_bound(len(zs))
    print("%s: z %s; sum z^2 %.1f / %d p %.3g; min spectrum p %.3g" % (label, np.round(zs, 2), chi, dof, p, min(ps)))
    assert np.max(np.abs(zs)) < bound
    assert p > 1e-3
    assert min(ps) > 1e-3 / len(ps)


def test_lines_oracle_matches_reference():
    """PMMA lines on Si at 500 eV, 6 landing points, oracle 8 batches of 500 vs the reference's 16 of 1000."""
    from cudamonsel_b200 import scenes
    ob, of, ref = oracle_batches("lines_points", scenes.lines(), 8, 500, 100)
    check(ob, of, ref, 500, "lines")


@pytest.mark.parametrize("name", ["si_mott2", "si_mott3", "pmma_mott2", "pmma_mott3", "si_phonon"])
def test_halfspace_oracle_matches_reference(name):
    """Flat Si/PMMA with NISTMottRS methods 2 and 3 (300 eV) and Si with the phonon mechanism (500 eV)."""
    from cudamonsel_b200 import scenes
    sc = {"si_mott2": lambda: scenes.halfspace(mott_method=2), "si_mott3": lambda: scenes.halfspace(mott_method=3),
          "pmma_mott2": lambda: scenes.halfspace(material="pmma", mott_method=2),
          "pmma_mott3": lambda: scenes.halfspace(material="pmma", mott_method=3),
          "si_phonon": lambda: scenes.halfspace(phonon=True)}[name]()
    ob, of, ref = oracle_batches(name, sc, 8, 2000, 200)
    check(ob, of, ref, 2000, name)


def test_family_bound_and_t_to_z():
    """The family-wise bound reduces to 3 for one comparison and grows with k; t converts to z by tail."""
    from cudamonsel_b200 import stats
    assert abs(stats.family_z_bound(1) - 3.0) < 1e-12
    assert 3.6 < stats.family_z_bound(12) < 3.8
    assert abs(float(stats.t_to_z(3.0, 10 ** 7)) - 3.0) < 1e-4
    assert float(stats.t_to_z(3.0, 10)) < 3.0
