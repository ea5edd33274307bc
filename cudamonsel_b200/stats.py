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


# ---------------------------------------------------------------- whole-run comparisons
def family_z_bound(k, sigmas=3.0):
    """|z| bound per comparison that gives a family of k independent comparisons the false-alarm
    probability of one two-sided comparison at `sigmas` standard errors (Sidak correction).
    k = 1 gives `sigmas` itself."""
    from scipy.stats import norm
    a = 2.0 * norm.sf(sigmas)
    ak = 1.0 - (1.0 - a) ** (1.0 / max(int(k), 1))
    return float(norm.isf(ak / 2.0))


def t_to_z(t, dof):
    """The standard-normal deviate with the same two-sided tail probability as Student's t."""
    from scipy.stats import norm, t as tdist
    t = np.asarray(t, dtype=np.float64)
    p = 2.0 * tdist.sf(np.abs(t), dof)
    return np.sign(t) * norm.isf(p / 2.0)


def pooled_z(a_batches, b_batches):
    """z of the difference of the means of two sets of equal-size batch values (yields of independent
    batches of the same number of primaries within each set), from the pooled per-batch variance
    (equal under the hypothesis that both sides sample the same process), as the normal equivalent
    of the pooled t statistic.  Returns (z, mean_a, mean_b, standard error of the difference)."""
    a = np.asarray(a_batches, dtype=np.float64)
    b = np.asarray(b_batches, dtype=np.float64)
    na, nb = len(a), len(b)
    ma, mb = a.mean(), b.mean()
    ssq = ((a - ma) ** 2).sum() + ((b - mb) ** 2).sum()
    dof = na + nb - 2
    var = ssq / dof
    se = math.sqrt(var * (1.0 / na + 1.0 / nb))
    if se == 0.0:
        return 0.0 if ma == mb else math.copysign(float("inf"), ma - mb), ma, mb, se
    return float(t_to_z((ma - mb) / se, dof)), ma, mb, se


def pooled_z_weighted(a_batches, na_prim, b_batches, nb_prim):
    """pooled_z for batches of different sizes on the two sides: per-primary variance pooled from both
    (a batch of n primaries has variance sigma1^2 / n)."""
    a = np.asarray(a_batches, dtype=np.float64)
    b = np.asarray(b_batches, dtype=np.float64)
    ma, mb = a.mean(), b.mean()
    dof = len(a) + len(b) - 2
    s1 = (((a - ma) ** 2).sum() * na_prim + ((b - mb) ** 2).sum() * nb_prim) / dof
    se = math.sqrt(s1 * (1.0 / (len(a) * na_prim) + 1.0 / (len(b) * nb_prim)))
    if se == 0.0:
        return 0.0 if ma == mb else math.copysign(float("inf"), ma - mb), ma, mb, se
    return float(t_to_z((ma - mb) / se, dof)), ma, mb, se


def chi2_of_z(z):
    """Sum of squared z over independent comparisons and its chi-squared tail probability."""
    from scipy.stats import chi2 as chi2dist
    z = np.asarray(z, dtype=np.float64).ravel()
    c = float((z * z).sum())
    return c, len(z), float(chi2dist.sf(c, len(z)))


def scan_z(a_batches, na, b_mean, nb):
    """Per-pixel z of a scan's yields: a_batches[B, npix] are side a's yields from B independent batches of
    na primaries per pixel, b_mean[npix] side b's yields from nb primaries per pixel.  Each pixel's
    variance comes from its own B batches (B - 1 degrees of freedom; under the hypothesis that both sides
    sample the same process it is side b's too), and z is the normal equivalent of the t statistic:
    a batch yield has variance v, a primary v * na, so the difference of the means has variance
    v * na * (1 / (B na) + 1 / nb) = v * (1 / B + na / nb)."""
    a = np.asarray(a_batches, dtype=np.float64)
    B = a.shape[0]
    v = a.var(0, ddof=1)
    se = np.sqrt(v * (1.0 / B + na / float(nb)))
    t = (a.mean(0) - np.asarray(b_mean, dtype=np.float64)) / np.maximum(se, 1e-300)
    return t_to_z(t, B - 1)


def repeats_z(a_runs, b_runs, nprim=None, groups=None, bins=32):
    """Per-pixel z between two sets of independent repeats of the same scan: a_runs[Ra, npix] and
    b_runs[Rb, npix] are per-pixel yields of runs on streams of their own (equal primaries per pixel
    within a pixel).

    Without nprim, each pixel's variance is pooled from its own repeats (Ra + Rb - 2 degrees of freedom)
    and z is the normal equivalent of the pooled t statistic.  With few repeats of counts that take few
    values this is fragile: repeats that happen to give the same count make the variance estimate zero.
    With nprim[npix], a pixel's variance is instead v(y) / nprim, the per-primary variance v taken as the
    mean of the pixels' own estimates (variance x nprim) over the pixels whose mean yield falls in the
    same of `bins` quantile bins (within the same group, e.g. the same beam energy, when groups[npix] is
    given): pixels of the same yield share a variance, estimated from thousands of degrees of freedom,
    and z is normal."""
    a = np.asarray(a_runs, dtype=np.float64)
    b = np.asarray(b_runs, dtype=np.float64)
    ra, rb = a.shape[0], b.shape[0]
    ma, mb = a.mean(0), b.mean(0)
    dof = ra + rb - 2
    var = (((a - ma) ** 2).sum(0) + ((b - mb) ** 2).sum(0)) / dof
    d = ma - mb
    if nprim is None:
        se = np.sqrt(var * (1.0 / ra + 1.0 / rb))
        t = np.where(se > 0, d / np.where(se > 0, se, 1.0), np.where(d == 0, 0.0, np.sign(d) * 1e300))
        return t_to_z(t, dof)
    n = np.broadcast_to(np.asarray(nprim, dtype=np.float64), d.shape)
    per_primary = var * n
    m = (ma * ra + mb * rb) / (ra + rb)
    g = np.zeros(d.shape, dtype=np.int64) if groups is None else np.unique(np.asarray(groups), return_inverse=True)[1]
    model = np.empty_like(per_primary)
    for k in np.unique(g):
        sel = np.nonzero(g == k)[0]
        edges = np.quantile(m[sel], np.linspace(0.0, 1.0, bins + 1))
        idx = np.clip(np.searchsorted(edges, m[sel], side="right") - 1, 0, bins - 1)
        cnt = np.bincount(idx, minlength=bins)
        mean = np.bincount(idx, weights=per_primary[sel], minlength=bins) / np.maximum(cnt, 1)
        model[sel] = mean[idx]
    se = np.sqrt(model / n * (1.0 / ra + 1.0 / rb))
    return np.where(se > 0, d / np.where(se > 0, se, 1.0), 0.0)


def z_summary(z):
    """What a per-pixel z map says: largest |z|, pixels beyond 3 and beyond the family-wise bound of
    3 standard errors for this many pixels, and the chi-squared of the sum of z^2."""
    z = np.asarray(z, dtype=np.float64).ravel()
    bound = family_z_bound(len(z))
    c, dof, p = chi2_of_z(z)
    return {"pixels": int(len(z)), "max_abs_z": float(np.abs(z).max()), "over_3": int((np.abs(z) > 3).sum()),
            "family_bound": bound, "over_family_bound": int((np.abs(z) > bound).sum()), "chi2": c, "dof": dof,
            "chi2_p": p}
