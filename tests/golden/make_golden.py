"""Regenerate the golden vectors from the reference itself.

Builds the reference's own CPU code out of tree (oracle/build_ref.py), runs
oracle/_ref/ref_driver in ``golden`` mode on the synthetic Si tables and
gzips the text files into tests/golden/.  Needs the reference checkout
(found by oracle/build_ref.py, $CM_REFERENCE_ROOT); the fixtures are committed.

    python tests/golden/make_golden.py
"""
import gzip
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "build_ref.py")])
    ref = os.path.join(ROOT, "oracle", "_ref")
    tables = os.path.join(ROOT, "cudamonsel_b200", "data", "ScatteringTables", "SiTables")
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.check_call([os.path.join(ref, "ref_driver"), "golden", tmp, tables], cwd=ref,
                              stdout=subprocess.DEVNULL)
        subprocess.check_call([os.path.join(ref, "ref_driver"), "golden2", tmp], cwd=ref, stdout=subprocess.DEVNULL)
        for name in sorted(os.listdir(tmp)):
            src = os.path.join(tmp, name)
            with open(src, "rb") as f, gzip.open(os.path.join(HERE, name + ".gz"), "wb", compresslevel=9) as g:
                shutil.copyfileobj(f, g)
            print("wrote", name + ".gz")
    # whole runs of the flat Si sample at 1 keV (pencil beam, 10 000 primaries, 4 seeds)
    out = []
    for seed in (11, 12, 13, 14):
        r = subprocess.run([os.path.join(ref, "ref_driver"), "run1", "10000", str(seed), tables, "1000"], cwd=ref,
                           capture_output=True, text=True, check=True)
        out.append("# seed %d\n" % seed + "\n".join(l for l in r.stdout.splitlines()
                                                    if l.startswith(("pixel", "back", "fwd", "elev", "azim", "steps",
                                                                       "seconds", "#"))))
    with open(os.path.join(HERE, "run_halfspace_1keV.txt"), "w") as f:
        f.write("\n".join(out) + "\n")
    print("wrote run_halfspace_1keV.txt")


if __name__ == "__main__":
    main()
