"""Scattering tables from a dielectric model (cudamonsel_b200/data/gen_penn_tables.py).

The model's energy-loss function obeys the f-sum rule; the Penn single-pole inverse mean free path
follows the TPP-2M formula for Si; tables in the reference's format load into the reference's own code,
the oracle and the engine, and whole runs on them agree (statistically) between the three.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


@pytest.fixture(scope="module")
def penn_dir(tmp_path_factory):
    from cudamonsel_b200.data import gen_penn_tables
    d = str(tmp_path_factory.mktemp("penn"))
    gen_penn_tables.build(d, n_iimfp=48, n_loss=24, n_theta=(16, 17, 17))
    return d


def test_energy_loss_function_sum_rule():
    from cudamonsel_b200.data import gen_penn_tables as p
    w = np.geomspace(0.5, 2e5, 400000)
    lhs = np.trapezoid(w * p.elf(w), w)
    rhs = np.pi / 2 * p.EP ** 2 * (1 + sum(n for _, n in p.SHELLS) / 4.0)  # 4 valence + 10 core electrons
    assert abs(lhs / rhs - 1) < 2e-3


def test_mean_free_path_follows_tpp2m():
    from cudamonsel_b200.data import gen_penn_tables as p
    for E in (50.0, 100.0, 300.0, 1000.0, 3000.0, 10000.0):
        lam = 1e9 / p.iimfp_per_m(E + p.g.OFFSET_FERMI)
        ratio = lam / p.tpp2m_imfp_nm(E)
        print("E %6.0f eV: Penn %.3f nm, TPP-2M %.3f nm" % (E, lam, p.tpp2m_imfp_nm(E)))
        assert 0.9 < ratio < 1.1


def test_tables_are_monotonic_inverse_cdfs(penn_dir):
    from cudamonsel_b200.data import gen_si_tables as g
    def read(name):
        v = np.array(open(os.path.join(penn_dir, name)).read().split(), dtype=np.float64)
        dim = int(v[0])
        axes, k = [], 1
        for _ in range(dim):
            n = int(v[k])
            axes.append(v[k + 1:k + 1 + n])
            k += 1 + n
        return axes, v[k:].reshape([len(a) for a in axes])
    _, iimfp = read(g.NAMES[0])
    (e2, r2), red = read(g.NAMES[1])
    (e3, q3, r3), th = read(g.NAMES[2])
    assert np.isfinite(iimfp).all() and (iimfp > 0).all()
    assert (np.diff(red, axis=1) >= 0).all() and (red >= 0).all() and (red <= 1).all()
    assert (np.diff(th, axis=2) >= -1e-12).all() and (th >= 0).all() and (th <= np.pi).all()
    # the mean loss at 1 keV sits near the valence plasmon (16.6 eV), far below the beam energy
    i = np.argmin(abs(e2 / g.EV - 1000.0))
    assert 12.0 < np.median(red[i]) * e2[i] / g.EV < 40.0


def _yields(back, nprim, beam_eV, nbins):
    from cudamonsel_b200 import scenes
    return scenes.yields(back, nprim, beam_eV, nbins)


def _ref_run(tables, seed, nprim=2000):
    r = subprocess.run([REF, "run1", str(nprim), str(seed), tables, "1000"], cwd=os.path.dirname(REF),
                       capture_output=True, text=True, check=True, timeout=300)
    return np.array([[int(x) for x in l.split()[1:]] for l in r.stdout.splitlines() if l.startswith("back")])


@pytest.mark.skipif(not os.path.exists(REF), reason="the reference's own code is built only where its sources are")
def test_oracle_matches_reference_on_penn_tables(penn_dir):
    """1 keV pencil beam on flat Si with the Penn tables: the reference's code (8 x 1500 primaries) and
    the oracle (8 x 1500) agree in BSE/SE yields and escape spectra."""
    import pyoracle
    from cudamonsel_b200 import scenes, stats
    from cudamonsel_b200.data import gen_si_tables as g
    tables = [os.path.join(penn_dir, n) for n in g.NAMES]
    ref = np.concatenate([_ref_run(penn_dir, s, 1500) for s in range(31, 39)])
    sc = scenes.halfspace(tables=tables)
    ob, _, _ = pyoracle.run_scene(sc, np.tile([0.0, 0.0, -20e-9], (8, 1)), 0.0, scenes.eV(1000.0), 1500, 41, 100)
    rb, rs = _yields(ref, 1500, 1000.0, 100)
    obb, os_ = _yields(ob, 1500, 1000.0, 100)
    print("BSE ref %.4f oracle %.4f | SE ref %.4f oracle %.4f" % (rb.mean(), obb.mean(), rs.mean(), os_.mean()))
    for a, b in ((rb, obb), (rs, os_)):
        se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
        assert abs(a.mean() - b.mean()) < 4.0 * max(se, 1e-4)
    _, _, p = stats.chi2_two_sample(ref.sum(0), 12000, ob.sum(0), 12000)
    assert p > 1e-3
