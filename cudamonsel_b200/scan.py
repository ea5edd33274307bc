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


def run_checkpointed(engine, chamber, centers, energies, nprim, nbins, beam_width, precision, pixel_keys, part=None,
                     checkpoint=None, max_parts=None):
    """A scan run in parts of at most `part` primaries per pixel, resumable.

    After each part the primaries done per pixel and the tallies so far are written to `checkpoint` (an .npz,
    replaced atomically); a call that finds the file carries on from it (its pixel keys and primary counts
    must be this scan's).  Primary k of a pixel draws from a stream keyed by (pixel key, k) -- the run's
    pixel_first is the primaries already done -- so the result equals that of one cm_run over the whole scan,
    count for count.  max_parts stops after that many parts (the checkpoint holds the rest).  Returns
    (back, fwd, done): uint64 tallies [npix, max(nbins) + 2] and the primaries done per pixel."""
    import os
    centers = np.asarray(centers, dtype=np.float64).reshape(-1, 3)
    npix = len(centers)
    keys = np.ascontiguousarray(pixel_keys, dtype=np.uint64)
    nprim = np.ascontiguousarray(np.broadcast_to(np.asarray(nprim), (npix,)), dtype=np.int64)
    stride = int(np.max(nbins)) + 2
    done = np.zeros(npix, dtype=np.int64)
    back = np.zeros((npix, stride), dtype=np.uint64)
    fwd = np.zeros((npix, stride), dtype=np.uint64)
    if checkpoint and os.path.exists(checkpoint):
        z = np.load(checkpoint)
        if not (np.array_equal(z["keys"], keys) and np.array_equal(z["nprim"], nprim) and z["back"].shape == back.shape):
            raise ValueError("checkpoint %s belongs to another scan" % checkpoint)
        done, back, fwd = z["done"].astype(np.int64), z["back"].astype(np.uint64), z["fwd"].astype(np.uint64)
    part = int(part or max(1, int(nprim.max())))
    parts = 0
    while (done < nprim).any() and (max_parts is None or parts < max_parts):
        todo = np.minimum(part, nprim - done)
        b, f, _ = engine.run(chamber, centers, energies, todo.astype(np.int32), nbins, beam_width, 0,
                             precision=precision, pixel_keys=keys, first_primary=done)
        back += b.astype(np.uint64)
        fwd += f.astype(np.uint64)
        done = done + todo
        parts += 1
        if checkpoint:
            tmp = checkpoint + ".tmp.npz"
            np.savez(tmp, keys=keys, nprim=nprim, done=done, back=back, fwd=fwd)
            os.replace(tmp, checkpoint)
    return back, fwd, done
