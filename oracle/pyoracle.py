"""ctypes front end of the C oracle (oracle/cm_oracle.c) -- test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the library never does.  It builds ``liboracle.so`` on first use
if gcc is available and the library is missing or stale.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "cm_oracle.c")

EV = 1.60217653e-19


def build(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    subprocess.check_call(["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-o", LIB, SRC, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        d = C.POINTER(C.c_double)
        i = C.POINTER(C.c_int)
        L.cmo_scene_new.restype = C.c_void_p
        L.cmo_scene_free.argtypes = [C.c_void_p]
        L.cmo_scene_set_options.argtypes = [C.c_void_p, C.c_int]
        L.cmo_add_mott_element.argtypes = [C.c_void_p, C.c_int, d, d]
        L.cmo_add_table_file.argtypes = [C.c_void_p, C.c_char_p]
        L.cmo_add_material.argtypes = [C.c_void_p, C.c_int, i, d, d, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_int, d]
        L.cmo_add_msm.argtypes = [C.c_void_p, C.c_int]
        L.cmo_msm_add_nistmott.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.cmo_msm_add_tabulated.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, i]
        L.cmo_msm_add_fitted.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        L.cmo_msm_add_phonon.argtypes = [C.c_void_p, C.c_int] + [C.c_double] * 5
        L.cmo_msm_add_polaron.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        L.cmo_msm_set_csd_jln.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.cmo_msm_set_min_e.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.cmo_msm_set_barrier.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double]
        L.cmo_shape_sphere.argtypes = [C.c_void_p, d, C.c_double]
        L.cmo_shape_planes.argtypes = [C.c_void_p, C.c_int, d, d]
        L.cmo_shape_intersection.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.cmo_shape_translate.argtypes = [C.c_void_p, C.c_int, d]
        L.cmo_shape_rotate.argtypes = [C.c_void_p, C.c_int, d, C.c_double, C.c_double, C.c_double]
        L.cmo_shape_line.argtypes = [C.c_void_p] + [C.c_double] * 7
        L.cmo_shape_cylinder.argtypes = [C.c_void_p, d, d, C.c_double]
        L.cmo_shape_union.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.cmo_region.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.cmo_eval_nistmott.argtypes = [C.c_void_p, C.c_int, C.c_int, d, d, d, d, i]
        L.cmo_eval_nistmott_method.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, d, d, d, d, i]
        L.cmo_eval_table.argtypes = [C.c_void_p, C.c_int, C.c_int, d, C.c_int, d]
        L.cmo_eval_tabulated.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, d, d]
        L.cmo_eval_tabulated_stride.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, d, d, C.c_int]
        L.cmo_table_window.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.cmo_table_locate.argtypes = [C.c_void_p, C.c_int, C.c_int, d, C.c_int, i]
        L.cmo_eval_pick.argtypes = [C.c_void_p, C.c_int, C.c_int, d, d]
        L.cmo_eval_elastic.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, d, d]
        L.cmo_eval_pmma.argtypes = [C.c_void_p, C.c_int, C.c_int, d, d]
        L.cmo_eval_phonon.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, d, d]
        L.cmo_eval_shape.argtypes = [C.c_void_p, C.c_int, C.c_int, d, d]
        L.cmo_eval_barrier.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, d, d]
        L.cmo_eval_freepath.argtypes = [C.c_void_p, C.c_int, C.c_int, d, d]
        L.cmo_eval_beam.argtypes = [C.c_int, d, d]
        L.cmo_hist_bin.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double]
        L.cmo_run.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, d, C.c_int, C.c_uint64, C.c_int,
                              C.c_void_p]
    return _lib


def dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def ip(a):
    return np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(C.POINTER(C.c_int))


class Tally(C.Structure):
    _fields_ = [("back", C.c_int64 * 1026), ("fwd", C.c_int64 * 1026), ("trajectories", C.c_int64),
                ("scatter_events", C.c_int64), ("barrier_events", C.c_int64), ("secondaries", C.c_int64),
                ("dropped_overrange", C.c_int64), ("elevation", C.c_int64 * 182), ("azimuth", C.c_int64 * 362)]


class Scene:
    """A scene description replayed into the C oracle (SI units throughout)."""

    def __init__(self, options=0):
        self.L = lib()
        self.h = C.c_void_p(self.L.cmo_scene_new())
        self.L.cmo_scene_set_options(self.h, options)
        self._keep = []

    def __del__(self):
        try:
            self.L.cmo_scene_free(self.h)
        except Exception:
            pass

    def _k(self, *arrs):
        out = [np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
        self._keep.extend(out)
        return out

    def mott(self, Z, spwem, x1):
        a, b = self._k(spwem, x1)
        return self.L.cmo_add_mott_element(self.h, Z, dp(a), dp(b))

    def table(self, path):
        t = self.L.cmo_add_table_file(self.h, path.encode())
        assert t >= 0, path
        return t

    def material(self, Z, A, wf, density, workfunction, ecb, bandgap, core=()):
        Zi = np.ascontiguousarray(Z, dtype=np.int32)
        a, w, c = self._k(A, wf, np.array(core, dtype=np.float64) if len(core) else np.zeros(1))
        return self.L.cmo_add_material(self.h, len(Z), Zi.ctypes.data_as(C.POINTER(C.c_int)), dp(a), dp(w),
                                       density, workfunction, ecb, bandgap, len(core), dp(c))

    def run(self, chamber, width, energy, center, nprim, seed, nbins):
        t = Tally()
        c = np.array(center, dtype=np.float64)
        rc = self.L.cmo_run(self.h, chamber, width, energy, dp(c), nprim, seed, nbins, C.byref(t))
        assert rc == 0
        return t


class OracleBackend:
    """Replays a cudamonsel_b200.scenes.SceneSpec into the C oracle (same call names)."""

    def __init__(self, options=0):
        self.s = Scene(options)
        self.L = self.s.L
        self.h = self.s.h

    def begin(self, spec):
        from cudamonsel_b200 import data
        self.L.cmo_scene_set_options(self.h, spec.options)
        for Z in sorted(spec.elements):
            spwem, x1 = data.read_mott(Z)
            self.s.mott(Z, spwem, x1)

    def set_options(self, options):
        self.L.cmo_scene_set_options(self.h, options)

    def _chk(self, v):
        assert v >= 0, "oracle scene call failed (%d)" % v
        return v

    def table(self, path):
        return self.s.table(path)

    def material(self, Z, A, wf, density, workfunction, ecb, bandgap, core=()):
        return self._chk(self.s.material(Z, A, wf, density, workfunction, ecb, bandgap, core))

    def msm(self, material):
        return self._chk(self.L.cmo_add_msm(self.h, material))

    def nistmott(self, msm, method=1):
        return self._chk(self.L.cmo_msm_add_nistmott(self.h, msm, method))

    def tabulated(self, msm, method_se, offset, tables):
        t = np.ascontiguousarray(tables, dtype=np.int32)
        return self._chk(self.L.cmo_msm_add_tabulated(self.h, msm, method_se, offset, ip(t)))

    def fitted(self, msm, e, b):
        return self._chk(self.L.cmo_msm_add_fitted(self.h, msm, e, b))

    def phonon(self, msm, *a):
        return self._chk(self.L.cmo_msm_add_phonon(self.h, msm, *a))

    def polaron(self, msm, p, x):
        return self._chk(self.L.cmo_msm_add_polaron(self.h, msm, p, x))

    def csd_jln(self, msm, b):
        return self.L.cmo_msm_set_csd_jln(self.h, msm, b)

    def min_e(self, msm, e):
        return self.L.cmo_msm_set_min_e(self.h, msm, e)

    def sphere(self, c, r):
        c = np.array(c, dtype=np.float64)
        return self._chk(self.L.cmo_shape_sphere(self.h, dp(c), r))

    def planes(self, normals, points):
        n = np.array(normals, dtype=np.float64)
        p = np.array(points, dtype=np.float64)
        return self._chk(self.L.cmo_shape_planes(self.h, len(n) // 3, dp(n), dp(p)))

    def intersection(self, a, b):
        return self._chk(self.L.cmo_shape_intersection(self.h, a, b))

    def translate(self, shape, d):
        d = np.array(d, dtype=np.float64)
        return self.L.cmo_shape_translate(self.h, shape, dp(d))

    def rotate(self, shape, pivot, phi, theta, psi):
        pv = np.array(pivot, dtype=np.float64)
        return self.L.cmo_shape_rotate(self.h, shape, dp(pv), phi, theta, psi)

    def line(self, topz, width, length, thetal, thetar, radl=0.0, radr=0.0):
        return self._chk(self.L.cmo_shape_line(self.h, topz, width, length, thetal, thetar, radl, radr))

    def cylinder(self, end0, end1, radius):
        return self._chk(self.L.cmo_shape_cylinder(self.h, dp(list(end0)), dp(list(end1)), radius))

    def union(self, a, b):
        return self._chk(self.L.cmo_shape_union(self.h, a, b))

    def region(self, parent, msm, shape):
        return self._chk(self.L.cmo_region(self.h, parent, msm, shape))


def build_oracle(scene):
    """Replay a cudamonsel_b200.scenes.Scene into the oracle; returns (backend, handles)."""
    from cudamonsel_b200.scenes import replay
    b = OracleBackend()
    res = replay(scene.spec, b)
    out = {"chamber": res[scene.chamber.idx]}
    for k, v in scene.h.items():
        out[k] = [res[x.idx] for x in v] if isinstance(v, list) else res[v.idx]
    return b, out


def run_scene(scene, centers, beam_width, beam_energy, nprim, seed, nbins):
    """Whole trajectories on the oracle for each landing point; returns (back[npix, nbins+2], fwd, tallies)."""
    b, h = build_oracle(scene)
    backs, fwds, tallies = [], [], []
    for i, c in enumerate(np.atleast_2d(centers)):
        t = b.s.run(h["chamber"], beam_width, beam_energy, c, nprim, seed + i, nbins)
        backs.append(np.array(t.back[:nbins + 2]))
        fwds.append(np.array(t.fwd[:nbins + 2]))
        tallies.append(t)
    return np.array(backs), np.array(fwds), tallies
