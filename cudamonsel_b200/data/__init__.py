"""Data files the transport path needs: NIST SRD-64 elastic tables and
NUTableInterpolation scattering tables (see gen_si_tables.py, pack_nistmott.py)."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SI_TABLES = os.path.join(HERE, "ScatteringTables", "SiTables")
SI_TABLE_NAMES = (
    "IIMFPFullPennInterpSiSI.csv",
    "interpNUSimReducedDeltaEFullPennSiSI.csv",
    "interpNUThetaFullPennSiBGSI.csv",
    "interpSimESE0NUSiBGSI.csv",
)

# Nominal atomic weights (g/mol) of the elements used by the standard scenes.
# The reference parses EPQLibrary/AtomicWeights.csv with std::stof
# (EPQLibrary/Element.cu:590-608), so each value is rounded to float.
_ATOMIC_WEIGHT_DEC = {1: "1.00794", 6: "12.0107", 7: "14.0067", 8: "15.9994", 13: "26.981538", 14: "28.0855",
                      29: "63.546", 79: "196.96655"}


def atomic_weight(Z):
    return float(np.float32(float(_ATOMIC_WEIGHT_DEC[Z])))


def si_tables(dirpath=SI_TABLES):
    return [os.path.join(dirpath, n) for n in SI_TABLE_NAMES]


def read_nu_table(path):
    """Parse a NUTableInterpolation text table (JMONSEL/NUTableInterpolation.cu:117-228).

    Returns (dim, n[], axes[], values ndarray with the last index fastest)."""
    with open(path) as f:
        tok = f.read().split()
    try:
        pos = 0
        dim = int(tok[pos]); pos += 1
        if not 1 <= dim <= 4:
            raise ValueError("dimension %d" % dim)
        n, axes = [], []
        for _ in range(dim):
            k = int(tok[pos]); pos += 1
            if k < 1 or pos + k > len(tok):
                raise ValueError("axis of %d points" % k)
            axes.append(np.array([float(t) for t in tok[pos:pos + k]], dtype=np.float64)); pos += k
            n.append(k)
        total = int(np.prod(n))
        if pos + total > len(tok):
            raise ValueError("%d values of %d" % (len(tok) - pos, total))
        vals = np.array([float(t) for t in tok[pos:pos + total]], dtype=np.float64).reshape(n)
    except (IndexError, ValueError) as e:
        # the reference throws on a table it cannot read (NUTableInterpolation.cu:121)
        raise ValueError("corrupt or truncated scattering table %s: %s" % (path, e)) from None
    return dim, n, axes, vals


def read_mott(Z, dirpath=None):
    """(spwem[61], x1[61,201]) for element Z from E%02d.bin (or a reference E%02d.D64)."""
    from .pack_nistmott import parse_d64, read_bin
    dirpath = dirpath or os.path.join(HERE, "NistXSec")
    b = os.path.join(dirpath, "E%02d.bin" % Z)
    if os.path.exists(b):
        z, spwem, x1 = read_bin(b)
    else:
        z, spwem, x1 = parse_d64(os.path.join(dirpath, "E%02d.D64" % Z))
    assert z == Z
    return spwem, x1
