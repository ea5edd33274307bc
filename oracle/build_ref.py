"""Build the reference's own CPU transport code (CudaMONSEL, master branch) from its
sources, out of tree, and link it with ``oracle/ref_driver.cpp``.

This is test infrastructure only: the resulting ``oracle/_ref/ref_driver``
binary produces the golden vectors under ``tests/golden/`` and times the
reference on the host.  Nothing in the library links or runs it.

The reference tree is never modified.  It is copied to a scratch directory
(``$CM_REF_WORK`` or /tmp/cm_ref_build) and these mechanical changes are made to
the copy so that g++ 13 accepts MSVC-flavoured sources:

 1. ``#include "a\\b\\c"`` -> ``#include "a/b/c"``; include names that differ only
    in letter case (EPQlibrary, SEMaterial.cuh, ...) get symlinks;
 2. a force-included compat header adds the standard headers MSVC pulls in
    implicitly, ``strtok_s``/``itoa``/``_UI32_MAX`` shims;
 3. the in-class explicit specialisations ``GetElementBy<...>`` in
    EPQLibrary/Composition.cuh (used only in comments) are dropped;
 4. ``const NISTMottScatteringAngle* mScatter[];`` in a header becomes an
    ``extern`` declaration;
 5. ``VectorXd& pos1 = <temporary>`` in MonteCarloSS::takeStep binds by value;
 6. Windows data paths ``".\\gov\\..."`` use '/' and are resolved from the copy;
 7. ``Math2::random()`` draws from a hook the driver sets (fixed deviate
    queue, or a seeded generator); the per-trajectory ``printf("%d\\n", i)``
    in ``runMultipleTrajectories`` is removed;
 8. ``Histogram::add`` (Utility/Histogram.cu:92-95) skips a bin index past the
    end of its count vector.  The reference writes there (a value above the
    top edge, e.g. an electron that gained energy from a negative interpolated
    loss) and corrupts the heap; the count is never read back either way.

Nothing else changes: the arithmetic under test is the reference's as written.

    python oracle/build_ref.py [--jobs N]
"""
import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: $CM_REFERENCE_ROOT, else where this build's container mounts it
REF_ROOT = os.environ.get("CM_REFERENCE_ROOT", "/root/reference")
REF = os.path.join(REF_ROOT, "CudaMONSEL", "CudaMONSEL")
OUT = os.path.join(HERE, "_ref")

COMPAT_H = r"""
#pragma once
#include <cstring>
#include <cstdlib>
#include <cstdio>
#include <cmath>
#include <climits>
#include <cfloat>
#include <vector>
#include <set>
#include <map>
#include <unordered_set>
#include <unordered_map>
#include <algorithm>
#include <sstream>
#include <iostream>
#include <fstream>
#include <stack>
#include <string>
#include <functional>
#include <chrono>
#include <ctime>
#define strtok_s strtok_r
#ifndef _UI32_MAX
#define _UI32_MAX 0xffffffffu
#endif
static inline char* itoa(int v, char* buf, int) { sprintf(buf, "%d", v); return buf; }
extern "C" double cm_ref_uniform(void);
"""

EXCLUDE_DIRS = ("EPQTests", "JMONSELTests")


def sources(root):
    out = []
    for d, _, files in os.walk(os.path.join(root, "gov")):
        if any(x in d for x in EXCLUDE_DIRS):
            continue
        for f in files:
            if (f.endswith(".cu") or f == "CSVReader.cpp") and "_GPU" not in f:
                out.append(os.path.join(d, f))
    out.append(os.path.join(root, "Amphibian", "Algorithm.cu"))
    out.append(os.path.join(root, "Amphibian", "Hasher.cu"))
    return sorted(out)


INC_RE = re.compile(r'^(\s*#\s*include\s*")([^"]*)(")', re.M)


def fix_includes(text):
    return INC_RE.sub(lambda m: m.group(1) + m.group(2).replace("\\", "/") + m.group(3), text)


def case_symlinks(root):
    """Create symlinks for include targets that exist only under another letter case."""
    want = set()
    for d, _, files in os.walk(root):
        for f in files:
            if f.endswith((".cu", ".cuh", ".h", ".cpp")):
                with open(os.path.join(d, f), errors="replace") as fh:
                    for m in INC_RE.finditer(fh.read()):
                        want.add(m.group(2))
    made = 0
    for inc in sorted(want):
        target = os.path.join(root, inc)
        if os.path.exists(target) or not inc.startswith("gov/"):
            continue
        # walk the path case-insensitively
        cur = root
        real = []
        ok = True
        for part in inc.split("/"):
            cand = os.path.join(cur, part)
            if os.path.exists(cand):
                cur = cand
                real.append(part)
                continue
            hits = [e for e in os.listdir(cur)] if os.path.isdir(cur) else []
            hits = [e for e in hits if e.lower() == part.lower()]
            if not hits:
                ok = False
                break
            link = os.path.join(cur, part)
            if not os.path.lexists(link):
                os.symlink(hits[0], link)
                made += 1
            cur = os.path.join(cur, hits[0])
        if not ok:
            print("warning: unresolved include", inc)
    return made


def patch_tree(src):
    for d, _, files in os.walk(src):
        for f in files:
            if not f.endswith((".cu", ".cuh", ".h", ".cpp")):
                continue
            p = os.path.join(d, f)
            with open(p, errors="replace") as fh:
                t = fh.read()
            t2 = fix_includes(t)
            # Windows-relative data paths -> forward slashes
            t2 = t2.replace('".\\\\gov\\\\', '"./gov/').replace("\\\\", "/") if '".\\\\gov' in t2 else t2
            if t2 != t:
                with open(p, "w") as fh:
                    fh.write(t2)
    comp = os.path.join(src, "gov/nist/microanalysis/EPQLibrary/Composition.cuh")
    t = open(comp).read()
    t = re.sub(r"\n\s*template<>\s*\n\s*Element::Element GetElementBy<[^>]*>\([^)]*\)\s*\{[^}]*\}", "\n", t)
    open(comp, "w").write(t)
    nm = os.path.join(src, "gov/nist/microanalysis/EPQLibrary/NISTMottScatteringAngle.cuh")
    t = open(nm).read()
    t = t.replace("const NISTMottScatteringAngle* mScatter[];", "extern const NISTMottScatteringAngle* mScatter[113];")
    open(nm, "w").write(t)
    mc = os.path.join(src, "gov/nist/microanalysis/NISTMonte/MonteCarloSS.cu")
    t = open(mc).read()
    t = t.replace("VectorXd& pos1 = mElectron->candidatePoint", "VectorXd pos1 = mElectron->candidatePoint")
    t = t.replace('            printf("%d\\n", i);\n', "")
    open(mc, "w").write(t)
    m2 = os.path.join(src, "gov/nist/microanalysis/Utility/Math2.cu")
    t = open(m2).read()
    old = "   double random()\n   {\n      return (double)rand() / RAND_MAX;\n   }"
    assert old in t, "Math2::random body not found"
    t = t.replace(old, "   double random()\n   {\n      return cm_ref_uniform();\n   }")
    open(m2, "w").write(t)
    hp = os.path.join(src, "gov/nist/microanalysis/Utility/Histogram.cu")
    t = open(hp).read()
    old = "      ++mCounts[bin(val) + 1];"
    assert old in t, "Histogram::add body not found"
    t = t.replace(old, "      { int b = bin(val) + 1; if (b < (int)mCounts.size()) ++mCounts[b]; }")
    open(hp, "w").write(t)
    with open(os.path.join(src, "cm_compat.h"), "w") as fh:
        fh.write(COMPAT_H)


def compile_one(args):
    src, obj, inc = args
    cmd = ["g++", "-O2", "-std=c++17", "-fpermissive", "-w", "-x", "c++", "-include",
           os.path.join(inc, "cm_compat.h"), "-I", inc, "-I", "/usr/local/cuda/include",
           "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stderr[-3000:]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--work", default=os.environ.get("CM_REF_WORK", "/tmp/cm_ref_build"))
    a = ap.parse_args()
    if not os.path.isdir(REF):
        print("reference tree not found at %s (set CM_REFERENCE_ROOT to the CudaMONSEL checkout); "
              "nothing to build" % REF_ROOT)
        return 0
    src = os.path.join(a.work, "src")
    objd = os.path.join(a.work, "obj")
    stamp = os.path.join(a.work, "patched.stamp")
    if not os.path.exists(stamp):
        shutil.rmtree(a.work, ignore_errors=True)
        shutil.copytree(REF, src, symlinks=True)
        patch_tree(src)
        case_symlinks(src)
        open(stamp, "w").write("ok")
    os.makedirs(objd, exist_ok=True)
    jobs = []
    for s in sources(src):
        rel = os.path.relpath(s, src).replace("/", "_")
        obj = os.path.join(objd, os.path.splitext(rel)[0] + ".o")
        if not os.path.exists(obj) or os.path.getmtime(obj) < os.path.getmtime(s):
            jobs.append((s, obj, src))
    fails = []
    with cf.ThreadPoolExecutor(a.jobs) as ex:
        for s, rc, err in ex.map(compile_one, jobs):
            if rc != 0:
                fails.append((s, err))
    for s, err in fails:
        print("FAILED", s, "\n", err)
    if fails:
        return 1
    os.makedirs(OUT, exist_ok=True)
    objs = sorted(os.path.join(objd, f) for f in os.listdir(objd) if f.endswith(".o"))
    drv_obj = os.path.join(a.work, "ref_driver.o")
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-fpermissive", "-w", "-x", "c++", "-include",
                        os.path.join(src, "cm_compat.h"), "-I", src, "-I", "/usr/local/cuda/include",
                        "-I", os.path.join(HERE, "..", "cudamonsel_b200", "csrc"),
                        "-c", os.path.join(HERE, "ref_driver.cpp"), "-o", drv_obj])
    if r.returncode:
        return 1
    exe = os.path.join(OUT, "ref_driver")
    r = subprocess.run(["g++", "-O2", "-o", exe, drv_obj] + objs + ["-lm"])
    if r.returncode:
        return 1
    # the reference resolves its data files relative to the working directory:
    # copy its data (not its sources) next to the binary so that it runs from there
    for d, _, files in os.walk(os.path.join(src, "gov")):
        for f in files:
            if f.endswith((".cu", ".cuh", ".h", ".cpp", ".txt")) or os.path.islink(os.path.join(d, f)):
                continue
            dst = os.path.join(OUT, os.path.relpath(d, src))
            os.makedirs(dst, exist_ok=True)
            shutil.copy2(os.path.join(d, f), os.path.join(dst, f))
    print("built", exe)
    return 0


if __name__ == "__main__":
    sys.exit(main())
