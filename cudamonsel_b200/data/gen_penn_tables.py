"""Silicon scattering tables for TabulatedInelasticSM from a dielectric model.

TabulatedInelasticSM (``JMONSEL/TabulatedInelasticSM.cu:209-459``) reads four tables:
the inverse inelastic mean free path IIMFP(kE), the reduced energy loss dE/kE (kE, r), the deflection
angle theta(kE, reduced loss, r) and the initial SE energy E0(dE, r), where r is a uniform deviate and
the reduced loss is (dE - gap) / (kE - E_F,offset - 2 gap) (``TabulatedInelasticSM.cu:233,260``).  The
reference's own tables (``IIMFPFullPennInterpSiSI.csv`` ...) were computed by JMONSEL's authors with the
full Penn algorithm and are not distributed with it.  This module computes the first three from a model of
silicon's optical energy-loss function (ELF) with the Penn algorithm in its single-pole form:

* Optical ELF Im[-1/eps(w)]: a Drude-Lorentz term for the 4 valence electrons (w0 = Ep = 16.6 eV, the
  free-electron plasmon energy of Si; width 3.5 eV; zero below the 1.1 eV gap) plus power-law edges for
  the L2,3 (99.8 eV, 6 electrons), L1 (149.7 eV, 2) and K (1839 eV, 2) shells, Im ~ w^-3.5 above each edge.
  Every term is scaled to the Bethe f-sum rule, int w Im[-1/eps] dw = (pi/2) Omega_p^2 with Omega_p^2 the
  plasma frequency squared of its electrons.
* Penn single-pole approximation: Im[-1/eps(q, w)] = (w'/w) Im[-1/eps(w')] with w' = w - q^2/2 (atomic
  units), i.e. each optical pole w_p disperses as w_p + q^2/2.
* Differential inverse mean free path of an electron of kinetic energy E (a.u.):
  dl^-1/dw = 1/(pi E) int_{q-}^{q+} dq/q Im[-1/eps(q, w)],  q+- = sqrt(2E) +- sqrt(2(E - w)).
  IIMFP = int dl^-1/dw over w in [gap, E - E_F,offset - gap]; the energy-loss table is the inverse CDF
  of dl^-1/dw; the angle table is the inverse CDF of the momentum transfer q at fixed w (weight
  Im[-1/eps(q, w)]/q), turned into the angle by q^2 = k^2 + k'^2 - 2 k k' cos(theta).
* The SE initial-energy table keeps the free-electron (sqrt density of states) model of gen_si_tables.

Units and layout are those of the reference's files (SI: J, 1/m, radians; ``NUTableInterpolation.cu:
117-228``).  The tables are deterministic.  Run:
    python -m cudamonsel_b200.data.gen_penn_tables <outdir>
"""
import os
import sys

import numpy as np

from . import gen_si_tables as g

HARTREE = 27.211386245988   # eV
BOHR = 0.529177210903e-10   # m
EP = 16.6                   # eV, valence plasmon energy of Si (free-electron, 4 electrons per atom)
VALENCE_WIDTH = 3.5         # eV
# core shells of Si: binding energy (eV) and electrons per atom
SHELLS = ((99.8, 6), (149.7, 2), (1839.0, 2))
CORE_POWER = 3.5


def elf(w):
    """Optical energy-loss function Im[-1/eps(w)] of the model, w in eV (array)."""
    w = np.asarray(w, dtype=np.float64)
    out = np.where(w > g.BANDGAP, EP ** 2 * VALENCE_WIDTH * w / ((EP ** 2 - w ** 2) ** 2 + (VALENCE_WIDTH * w) ** 2), 0.0)
    for e, n in SHELLS:
        omega2 = EP ** 2 * n / 4.0  # plasma frequency squared of the shell's electrons
        b = 1.5 * (np.pi / 2.0) * omega2 / e ** 2
        out = out + np.where(w >= e, b * (e / np.maximum(w, e)) ** CORE_POWER, 0.0)
    return out


def _elf_au(w_au):
    return elf(w_au * HARTREE)


def _q_weights(E, w, nq=400):
    """Nodes q (a.u.) and weights of int_{q-}^{q+} dq/q Im[-1/eps(q, w)] for one (E, w) in a.u."""
    k, kp = np.sqrt(2.0 * E), np.sqrt(2.0 * (E - w))
    qlo, qhi = k - kp, min(k + kp, np.sqrt(2.0 * w))  # above sqrt(2w) the pole lies below zero energy
    if qhi <= qlo:
        return None, None
    q = np.geomspace(qlo, qhi, nq)
    wp = w - 0.5 * q * q
    f = (wp / w) * _elf_au(wp) / q
    return q, f


def diimfp(E_eV, w_eV, nq=400):
    """dl^-1/dw in 1/(m eV) at kinetic energy E and loss w (scalars, eV)."""
    E, w = E_eV / HARTREE, w_eV / HARTREE
    q, f = _q_weights(E, w, nq)
    if q is None:
        return 0.0
    val = np.trapezoid(f, q) / (np.pi * E)          # 1/(a0 Hartree)
    return val / BOHR / HARTREE


def loss_grid(kE_eV, n=1200):
    wmin = g.BANDGAP
    wmax = kE_eV - g.OFFSET_FERMI - g.BANDGAP
    return np.geomspace(wmin, wmax, n)


def iimfp_per_m(kE_eV):
    w = loss_grid(kE_eV)
    p = np.array([diimfp(kE_eV, x) for x in w])
    return np.trapezoid(p, w)


def reduced_delta_e(kE_eV, r):
    w = loss_grid(kE_eV)
    p = np.array([diimfp(kE_eV, x) for x in w])
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (p[1:] + p[:-1]) * np.diff(w))])
    cdf /= cdf[-1]
    return np.interp(r, cdf, w) / kE_eV


def theta_of(kE_eV, reduced, r):
    """Deflection angles (rad) at the deviates r for the loss of the given reduced energy."""
    dE = g.BANDGAP + reduced * (kE_eV - g.OFFSET_FERMI - 2.0 * g.BANDGAP)
    E, w = kE_eV / HARTREE, dE / HARTREE
    q, f = _q_weights(E, w)
    k, kp = np.sqrt(2.0 * E), np.sqrt(2.0 * (E - w))
    if q is None or not np.trapezoid(f, q) > 0:
        # no pole reaches this loss (it lies within the gap of every q): minimum momentum transfer
        qs = np.full_like(np.asarray(r, dtype=np.float64), k - kp)
        return np.arccos(np.clip((k * k + kp * kp - qs * qs) / (2.0 * k * kp), -1.0, 1.0))
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (f[1:] + f[:-1]) * np.diff(q))])
    cdf /= cdf[-1]
    qs = np.interp(r, cdf, q)
    return np.arccos(np.clip((k * k + kp * kp - qs * qs) / (2.0 * k * kp), -1.0, 1.0))


def tpp2m_imfp_nm(E_eV, rho=2.33, M=28.0855, nv=4, eg=1.1):
    """The TPP-2M predictive formula for the inelastic mean free path (nm), the yardstick of the tests."""
    ep = 28.8 * np.sqrt(nv * rho / M)
    u = nv * rho / M
    beta = -0.10 + 0.944 / np.sqrt(ep ** 2 + eg ** 2) + 0.069 * rho ** 0.1
    gamma = 0.191 / np.sqrt(rho)
    c = 1.97 - 0.91 * u
    d = 53.4 - 20.8 * u
    lam_angstrom = E_eV / (ep ** 2 * (beta * np.log(gamma * E_eV) - c / E_eV + d / E_eV ** 2))
    return lam_angstrom / 10.0


def build(outdir, n_iimfp=150, n_loss=60, n_theta=(40, 33, 33)):
    os.makedirs(outdir, exist_ok=True)
    paths = [os.path.join(outdir, n) for n in g.NAMES]
    e1 = np.geomspace(g.E_MIN, g.E_MAX, n_iimfp)
    g.write_table(paths[0], [e1 * g.EV], np.array([iimfp_per_m(e) for e in e1]))
    e2 = np.geomspace(g.E_MIN, g.E_MAX, n_loss)
    r2 = np.linspace(0.0, 1.0, 65)
    g.write_table(paths[1], [e2 * g.EV, r2], np.array([reduced_delta_e(e, r2) for e in e2]))
    e3 = np.geomspace(g.E_MIN, g.E_MAX, n_theta[0])
    q3 = np.linspace(0.0, 1.0, n_theta[1])
    r3 = np.linspace(0.0, 1.0, n_theta[2])
    g.write_table(paths[2], [e3 * g.EV, q3, r3], np.array([[theta_of(e, q, r3) for q in q3] for e in e3]))
    d4 = np.geomspace(g.BANDGAP, g.E_MAX, 64)
    r4 = np.linspace(0.0, 1.0, 33)
    g.write_table(paths[3], [d4 * g.EV, r4], np.array([[g.se_e0(d, r) for r in r4] for d in d4]) * g.EV)
    return paths


if __name__ == "__main__":
    for p in build(sys.argv[1]):
        print(p, os.path.getsize(p))
