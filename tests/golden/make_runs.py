"""Whole runs of the reference's own CPU code on the test scenes, written as fixtures.

Each set replays a scene of cudamonsel_b200.scenes through the reference's classes
(oracle/_ref/ref_driver ``scene`` mode, built by oracle/build_ref.py) in independent
batches: one process per batch, each with its own seed, all landing points of the set in
turn.  The outputs are the reference's BackscatterStats energy histograms per pixel
(back and forward, counts(-1..nbins)), gzipped into tests/golden/runs_<set>.txt.gz:

    # set <name> batch <b> seed <s>
    pixel x y z nprim
    back c(-1) c(0) ... c(nbins)
    fwd  ...

Needs the reference checkout; the fixtures are committed and read by the GPU tests.

    python tests/golden/make_runs.py [set ...]
"""
import concurrent.futures as cf
import gzip
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cudamonsel_b200 import scenes  # noqa: E402

LINE_XS = [-60e-9, -22e-9, -19e-9, -12e-9, 0.0, 100e-9]
ROUGH_XS = [-219e-9, -200e-9, -180e-9, -21e-9, 1e-9, 21e-9]
FEATURE_REF_XS = [-180e-9, -150e-9, -125e-9, -20e-9, 0.0, 150e-9]
DEEP_XS = [(-480e-9, -160e-9), (-160e-9, 160e-9), (160e-9, -160e-9), (480e-9, 160e-9)]


def _points(xs, z=-120e-9, ys=None):
    ys = ys if ys is not None else [0.0] * len(xs)
    return [(x, y, z) for x, y in zip(xs, ys)]


def sets():
    """name -> (scene builder, landing points, beam eV, nbins, beam width m, primaries per pixel per batch,
    batches, first seed, pixels per batch process (None: all))."""
    deep_sc = lambda: scenes.deep_features(seed=3, cells=4, cell=320e-9)[0]
    deep_top = scenes.deep_features(seed=3, cells=4, cell=320e-9)[1]
    lin = scenes.linescan_pixels(256, 1e-9, 0.0, -120e-9)
    return {
        "lines_points": (scenes.lines, _points(LINE_XS), 500.0, 50, 1e-9, 1000, 16, 1000, None),
        "linescan": (scenes.lines, [tuple(p) for p in lin], 500.0, 50, 1e-9, 2000, 1, 2000, 8),
        "rough_points": (lambda: scenes.rough_lines(seed=4),
                         _points(ROUGH_XS, ys=list(np.linspace(-40e-9, 40e-9, 6))), 500.0, 50, 1e-9, 1000, 16, 3000,
                         None),
        "features_ref_points": (scenes.features_ref, _points(FEATURE_REF_XS), 800.0, 80, 1e-9, 1000, 16, 4000, None),
        "deep_points": (deep_sc, [(x, y, -(deep_top + 20e-9)) for x, y in DEEP_XS], 10000.0, 1000, 1e-9, 250, 16,
                        5000, None),
        "si_mott2": (lambda: scenes.halfspace(mott_method=2), [(0.0, 0.0, -20e-9)], 300.0, 30, 0.0, 2000, 16, 6000,
                     None),
        "si_mott3": (lambda: scenes.halfspace(mott_method=3), [(0.0, 0.0, -20e-9)], 300.0, 30, 0.0, 2000, 16, 6100,
                     None),
        "pmma_mott2": (lambda: scenes.halfspace(material="pmma", mott_method=2), [(0.0, 0.0, -20e-9)], 300.0, 30,
                       0.0, 2000, 16, 6200, None),
        "pmma_mott3": (lambda: scenes.halfspace(material="pmma", mott_method=3), [(0.0, 0.0, -20e-9)], 300.0, 30,
                       0.0, 2000, 16, 6300, None),
        "si_phonon": (lambda: scenes.halfspace(phonon=True), [(0.0, 0.0, -20e-9)], 500.0, 50, 0.0, 2000, 16, 7000,
                      None),
    }


def _run(args):
    exe, scene_txt, px_txt, seed, width = args
    r = subprocess.run([exe, "scene", scene_txt, px_txt, str(seed), repr(width)], cwd=os.path.dirname(exe),
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference run failed (%d): %s" % (r.returncode, r.stderr[-500:]))
    keep = [l for l in r.stdout.splitlines() if l.startswith(("pixel", "back", "fwd", "steps", "seconds"))]
    return keep


def make(name, spec, exe, tmp, jobs):
    build, pts, beam_eV, nbins, width, nprim, batches, seed0, chunk = spec
    scene_txt = os.path.join(tmp, name + ".scene")
    with open(scene_txt, "w") as f:
        f.write(build().spec.to_text())
    chunk = chunk or len(pts)
    work = []
    for b in range(batches):
        for c0 in range(0, len(pts), chunk):
            px_txt = os.path.join(tmp, "%s_%d_%d.px" % (name, b, c0))
            with open(px_txt, "w") as f:
                for (x, y, z) in pts[c0:c0 + chunk]:
                    f.write("%r %r %r %r %d %d\n" % (float(x), float(y), float(z), float(scenes.eV(beam_eV)),
                                                      nprim, nbins))
            seed = seed0 + b * 1000 + c0
            work.append(((b, seed), (exe, scene_txt, px_txt, seed, width)))
    with cf.ThreadPoolExecutor(jobs) as ex:
        outs = list(ex.map(_run, [w[1] for w in work]))
    secs = 0.0
    lines = ["# set %s beam_eV %r nbins %d width %r nprim %d batches %d" % (name, beam_eV, nbins, width, nprim,
                                                                         batches)]
    for (b, seed), out in zip([w[0] for w in work], outs):
        lines.append("# set %s batch %d seed %d" % (name, b, seed))
        lines += [l for l in out if not l.startswith("seconds")]
        secs += sum(float(l.split()[1]) for l in out if l.startswith("seconds"))
    path = os.path.join(HERE, "runs_%s.txt.gz" % name)
    with gzip.open(path, "wt", compresslevel=9) as g:
        g.write("\n".join(lines) + "\n")
    print("wrote %s (%d processes, %.1f core-s of reference transport)" % (os.path.basename(path), len(work), secs))


def main():
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "build_ref.py")])
    if not os.path.exists(exe):
        print("the reference is not built (no checkout); fixtures left as they are")
        return 1
    want = sys.argv[1:] or list(sets())
    all_sets = sets()
    with tempfile.TemporaryDirectory() as tmp:
        for name in want:
            make(name, all_sets[name], exe, tmp, os.cpu_count() or 4)
    return 0


def load(name):
    """Parse a fixture: dict(beam_eV, nbins, width, nprim, batches, centers[npix, 3],
    back[batches, npix, nbins + 2], fwd[...]) with pixels in the order they were run."""
    path = os.path.join(HERE, "runs_%s.txt.gz" % name)
    meta = {}
    per = {}
    cur = None
    with gzip.open(path, "rt") as f:
        for line in f:
            w = line.split()
            if not w:
                continue
            if w[0] == "#" and "beam_eV" in w:
                meta = {"beam_eV": float(w[4]), "nbins": int(w[6]), "width": float(w[8]), "nprim": int(w[10]),
                        "batches": int(w[12])}
            elif w[0] == "#" and "batch" in w:
                cur = per.setdefault(int(w[4]), {"c": [], "back": [], "fwd": []})
            elif w[0] == "pixel":
                cur["c"].append([float(x) for x in w[1:4]])
            elif w[0] in ("back", "fwd"):
                cur[w[0]].append([int(x) for x in w[1:]])
    bs = sorted(per)
    meta["centers"] = np.array(per[bs[0]]["c"])
    meta["back"] = np.array([per[b]["back"] for b in bs], dtype=np.int64)
    meta["fwd"] = np.array([per[b]["fwd"] for b in bs], dtype=np.int64)
    return meta


if __name__ == "__main__":
    sys.exit(main())
