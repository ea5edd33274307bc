"""Synthetic silicon scattering tables for TabulatedInelasticSM.

The reference reads four tables for silicon from JMONSEL's distribution
(``JMONSELTests/LinesOnLayers.cu:187-193``: IIMFPFullPennInterpSiSI.csv,
interpNUSimReducedDeltaEFullPennSiSI.csv, interpNUThetaFullPennSiBGSI.csv,
interpSimESE0NUSiBGSI.csv).  Those files are not shipped with the reference,
so this script writes stand-ins with the same names, the same layout and the
same units (SI: joules, 1/m, radians), built from simple closed-form physics:

* IIMFP(kE): 1/lambda with lambda[nm] = 143/E'^2 + 0.082*sqrt(E'), E' = kE - E_F,offset
  (a universal-curve shape with its minimum near 60-80 eV).
* ReducedDeltaE(kE, r): inverse CDF of a Drude loss function (plasmon at 16.7 eV,
  width 4 eV) plus a 1/w^2 tail, on [gap, kE - E_F,offset - gap], divided by kE.
* Theta(kE, reduced, r): inverse CDF of the dipole distribution
  p(theta) ~ theta/(theta^2 + theta_E^2), theta_E = dE/(2 kE), cut at
  max(sqrt(dE/kE), 2 theta_E) (and at pi/2).
* SE E0(dE, r): initial SE energy above the band bottom with a sqrt density of
  states on [max(0, E_F,offset - dE), E_F,offset].

The table format is the one ``NUTableInterpolation::ReadTable`` parses
(``JMONSEL/NUTableInterpolation.cu:117-228``): whitespace-separated numbers:
dim, then for each input variable its count and monotonic values, then the
table values with the last index varying fastest.

Everything is deterministic (no random numbers).  Run:
    python -m cudamonsel_b200.data.gen_si_tables [outdir]
"""
import os
import sys

import numpy as np

EV = 1.60217653e-19  # J per eV, PhysicalConstants::ElectronCharge

# Silicon as LinesOnLayers.cu:172-196 sets it up
BANDGAP = 1.1
ENERGY_OFFSET = 13.54
EFERMI = -BANDGAP                      # SEmaterial::getEFermi = -E_CB - W = -(-3.75) - 4.85
OFFSET_FERMI = EFERMI + ENERGY_OFFSET  # TabulatedInelasticSM::setMaterial:472

E_MIN = 16.0      # eV, lowest kE in the energy tables (tracked electrons have kE >= 17.29 eV)
E_MAX = 20000.0   # eV

PLASMON = 16.7
PLASMON_WIDTH = 4.0
TAIL = 0.02

NAMES = (
    "IIMFPFullPennInterpSiSI.csv",
    "interpNUSimReducedDeltaEFullPennSiSI.csv",
    "interpNUThetaFullPennSiBGSI.csv",
    "interpSimESE0NUSiBGSI.csv",
)


def _fmt(values):
    return "\n".join("%.17g" % v for v in np.asarray(values, dtype=np.float64).ravel())


def write_table(path, axes, values):
    values = np.asarray(values, dtype=np.float64)
    assert values.shape == tuple(len(a) for a in axes)
    parts = [str(len(axes))]
    for a in axes:
        parts.append(str(len(a)))
        parts.append(_fmt(a))
    parts.append(_fmt(values))
    with open(path, "w") as f:
        f.write("\n".join(parts) + "\n")


def iimfp_per_m(kE_eV):
    ep = kE_eV - OFFSET_FERMI
    lam_nm = 143.0 / ep ** 2 + 0.082 * np.sqrt(ep)
    return 1e9 / lam_nm


def loss_pdf(w):
    drude = PLASMON_WIDTH * w * PLASMON ** 2 / ((w ** 2 - PLASMON ** 2) ** 2 + (PLASMON_WIDTH * w) ** 2)
    return drude + TAIL * (PLASMON / w) ** 2


def reduced_delta_e(kE_eV, r):
    wmin = BANDGAP
    wmax = kE_eV - OFFSET_FERMI - BANDGAP
    w = np.geomspace(wmin, wmax, 4001)
    p = loss_pdf(w)
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (p[1:] + p[:-1]) * np.diff(w))])
    cdf /= cdf[-1]
    return np.interp(r, cdf, w) / kE_eV


def theta_of(kE_eV, reduced, r):
    dE = BANDGAP + reduced * (kE_eV - OFFSET_FERMI - 2.0 * BANDGAP)
    thE = dE / (2.0 * kE_eV)
    thc = min(max(np.sqrt(dE / kE_eV), 2.0 * thE), np.pi / 2)
    return thE * np.sqrt((1.0 + (thc / thE) ** 2) ** r - 1.0)


def se_e0(dE_eV, r):
    hi = OFFSET_FERMI
    lo = max(0.0, OFFSET_FERMI - dE_eV)
    return (lo ** 1.5 + r * (hi ** 1.5 - lo ** 1.5)) ** (2.0 / 3.0)


def build(outdir):
    os.makedirs(outdir, exist_ok=True)
    # 1-D inverse inelastic mean free path
    e1 = np.geomspace(E_MIN, E_MAX, 150)
    write_table(os.path.join(outdir, NAMES[0]), [e1 * EV], iimfp_per_m(e1))
    # 2-D reduced energy loss
    e2 = np.geomspace(E_MIN, E_MAX, 60)
    r2 = np.linspace(0.0, 1.0, 65)
    red = np.array([reduced_delta_e(e, r2) for e in e2])
    write_table(os.path.join(outdir, NAMES[1]), [e2 * EV, r2], red)
    # 3-D scattering angle
    e3 = np.geomspace(E_MIN, E_MAX, 40)
    q3 = np.linspace(0.0, 1.0, 33)
    r3 = np.linspace(0.0, 1.0, 33)
    th = np.array([[[theta_of(e, q, r) for r in r3] for q in q3] for e in e3])
    write_table(os.path.join(outdir, NAMES[2]), [e3 * EV, q3, r3], th)
    # 2-D SE initial energy
    d4 = np.geomspace(BANDGAP, E_MAX, 64)
    r4 = np.linspace(0.0, 1.0, 33)
    e0 = np.array([[se_e0(d, r) for r in r4] for d in d4])
    write_table(os.path.join(outdir, NAMES[3]), [d4 * EV, r4], e0 * EV)
    return [os.path.join(outdir, n) for n in NAMES]


if __name__ == "__main__":
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ScatteringTables", "SiTables")
    for p in build(sys.argv[1] if len(sys.argv) > 1 else here):
        print(p, os.path.getsize(p))
