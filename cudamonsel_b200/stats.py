"""Statistics used to state the error of a transport result against another.

Yields are tallied as in LinesOnLayers.cu:366-376 (see scenes.yields).  One
primary can contribute several escapes (its secondaries), so the standard
error of a yield is estimated from independent batches (pixels or seeds run
with the same beam) rather than from a binomial formula.
"""
import math

import numpy as np


def batch_mean_se(values, weights=None):
    """Mean of per-batch values and its standard error (batches of equal size when weights is None)."""
    v = np.asarray(values, dtype=np.float64)
    w = np.ones_like(v) if weights is None else np.asarray(weights, dtype=np.float64)
    m = np.sum(w * v) / np.sum(w)
    if len(v) < 2:
        return m, float("nan")
    var = np.sum(w * (v - m) ** 2) / (np.sum(w) - np.sum(w ** 2) / np.sum(w))
    return m, math.sqrt(var * np.sum(w ** 2)) / np.sum(w)


def z_score(a_values, b_values):
    """(mean_a - mean_b) / combined standard error for two sets of independent batches."""
    ma, sa = batch_mean_se(a_values)
    mb, sb = batch_mean_se(b_values)
    return (ma - mb) / math.sqrt(sa * sa + sb * sb)


def chi2_two_sample(h1, n1, h2, n2, min_count=10):
    """Two-sample chi-squared test of two count histograms normalised to n1 and n2 trials.

    Bins with fewer than min_count expected counts in either sample are merged into
    their neighbour.  Returns (chi2, dof, p)."""
    from scipy.stats import chi2 as chi2dist
    a = np.asarray(h1, dtype=np.float64)
    b = np.asarray(h2, dtype=np.float64)
    # merge sparse bins left to right
    ma, mb, ca, cb = [], [], 0.0, 0.0
    for x, y in zip(a, b):
        ca += x
        cb += y
        if ca >= min_count and cb >= min_count:
            ma.append(ca)
            mb.append(cb)
            ca = cb = 0.0
    if (ca or cb) and ma:
        ma[-1] += ca
        mb[-1] += cb
    ma = np.array(ma)
    mb = np.array(mb)
    if len(ma) < 2:
        return 0.0, 0, 1.0
    k1 = math.sqrt(n2 / n1)
    k2 = math.sqrt(n1 / n2)
    chi = float(np.sum((k1 * ma - k2 * mb) ** 2 / (ma + mb)))
    dof = len(ma) - 1
    return chi, dof, float(chi2dist.sf(chi, dof))


def compare_spectra(h1, n1, h2, n2):
    return chi2_two_sample(h1, n1, h2, n2)[2]


def yield_z(back1, n1, back2, n2, beam_eV, nbins, overdispersion=None):
    """z-scores of BSE and SE yields between two summed back-hemisphere histograms.

    Without batches, the per-primary variance is taken from the counts (Poisson)
    times an overdispersion factor for the clustering of secondaries (default 2.5
    for SE, 1 for BSE)."""
    from .scenes import yields
    b1, s1 = yields(back1, n1, beam_eV, nbins)
    b2, s2 = yields(back2, n2, beam_eV, nbins)
    od_b, od_s = (1.0, 2.5) if overdispersion is None else overdispersion
    vb = od_b * (b1[0] / n1 + b2[0] / n2)
    vs = od_s * (s1[0] / n1 + s2[0] / n2)
    return (b1[0] - b2[0]) / math.sqrt(vb), (s1[0] - s2[0]) / math.sqrt(vs)
