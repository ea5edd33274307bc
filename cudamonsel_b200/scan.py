"""Scan read-out in the reference's output formats.

LinesOnLayers::run (JMONSELTests/LinesOnLayers.cu:330-398) writes a text file: a header of `# ...` and
`key: value` lines, the column line `beamE (eV)\tx(nm)\ty (nm)\tBSE yield\tSE yield`, one line per landing
point with the five numbers formatted by std::to_string (printf "%f"), and finally the elapsed seconds.
The yields are computed as there: SE = the counts of the bins below 50 eV over the trajectories (a float
ratio), BSE = the backscattered fraction minus SE.  An image is written as 8-bit PGM (the reference's
ImageUtil writes a BMP through Windows GDI; PGM is the headless equivalent) or as a .npy array.
"""
import numpy as np

from . import scenes


def to_string(x):
    """std::to_string of a double or an int."""
    if isinstance(x, (int, np.integer)):
        return "%d" % x
    return "%f" % x


def yields(back, nprim, beam_eV, nbins):
    """(BSE, SE) yields per landing point, as LinesOnLayers.cu:366-376 computes them from BackscatterStats."""
    return scenes.yields(back, nprim, beam_eV, nbins)


def output_text(rows, header=(), elapsed_s=None):
    """The reference's output.txt.  rows: iterable of (beamE_eV, x_nm, y_nm, bse, se); header: lines
    written after a leading newline, before the column line (e.g. "# Trajectories at each landing
    position: 100", "Line height (nm): 100.000000")."""
    out = "".join("\n" + h for h in header)
    out += "\n\nbeamE (eV)\tx(nm)\ty (nm)\tBSE yield\tSE yield"
    for e, x, y, b, s in rows:
        out += "\n" + " ".join(to_string(v) for v in (float(e), float(x), float(y), float(b), float(s)))
    if elapsed_s is not None:
        out += "\n" + to_string(float(elapsed_s))
    return out


def scan_rows(back, centers_m, beam_eV, nprim, nbins):
    """Rows (beamE eV, x nm, y nm, BSE, SE) of a scan from its tallies and landing points."""
    centers_m = np.asarray(centers_m, dtype=np.float64).reshape(-1, 3)
    beam_eV = np.broadcast_to(np.asarray(beam_eV, dtype=np.float64), (len(centers_m),))
    bse, se = yields(back, nprim, beam_eV, nbins)
    return [(beam_eV[i], centers_m[i, 0] * 1e9, centers_m[i, 1] * 1e9, bse[i], se[i]) for i in range(len(centers_m))]


def write_output(path, rows, header=(), elapsed_s=None):
    with open(path, "w") as f:
        f.write(output_text(rows, header, elapsed_s))


def write_pgm(path, image, lo=None, hi=None):
    """An 8-bit binary PGM of a 2-D array, scaled linearly from [lo, hi] (default: its range) to 0..255."""
    a = np.asarray(image, dtype=np.float64)
    lo = float(a.min()) if lo is None else lo
    hi = float(a.max()) if hi is None else hi
    g = np.zeros(a.shape, dtype=np.uint8) if hi <= lo else np.clip((a - lo) / (hi - lo) * 255.0 + 0.5, 0, 255).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(b"P5\n%d %d\n255\n" % (a.shape[1], a.shape[0]))
        f.write(g.tobytes())


def read_pgm(path):
    with open(path, "rb") as f:
        data = f.read()
    parts = data.split(b"\n", 3)
    w, h = (int(v) for v in parts[1].split())
    return np.frombuffer(parts[3], dtype=np.uint8).reshape(h, w)
