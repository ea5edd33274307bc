"""ctypes binding of the C ABI in include/cudamonsel_b200.h.

The shared library is built in-tree (``python -m cudamonsel_b200.build``).
There is no fallback: if the library is missing or no sm_100 device is
present, creating an Engine raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libcudamonsel_b200.so")

PREC_FP64 = 0
PREC_FP32 = 1
OPT_JMONSEL_FIXES = 1
OPT_EXACT_CSG = 2
OPT_SCAN_CHILDREN = 4
OPT_QUEUE_STEPS = 8
OPT_GLOBAL_TABLES = 16
# CM_E* statuses (include/cudamonsel_b200.h)
EINVAL, ECUDA, ENOMEM, ESTATE, EOVERFLOW, ELIMIT, ECANCELED, ETIMEOUT = -1, -2, -3, -4, -5, -6, -7, -8

# every symbol include/cudamonsel_b200.h declares
EXPORTS = (
    "cm_context_create", "cm_context_destroy", "cm_context_reset", "cm_last_error", "cm_set_options", "cm_version",
    "cm_data_dir",
    "cm_add_mott_element", "cm_add_table", "cm_add_material", "cm_add_msm", "cm_msm_add_nistmott",
    "cm_msm_add_tabulated", "cm_msm_add_fitted", "cm_msm_add_phonon", "cm_msm_add_polaron", "cm_msm_set_csd_jln",
    "cm_msm_set_min_e", "cm_msm_set_barrier", "cm_shape_sphere", "cm_shape_planes", "cm_shape_intersection",
    "cm_shape_union", "cm_shape_cylinder", "cm_shape_translate", "cm_shape_rotate", "cm_shape_line", "cm_region_add", "cm_run", "cm_run_device", "cm_run_noalloc",
    "cm_eval_nistmott", "cm_eval_table", "cm_eval_locate", "cm_eval_pick", "cm_eval_tabulated", "cm_eval_elastic", "cm_eval_csd", "cm_eval_phonon",
    "cm_eval_shape", "cm_eval_barrier", "cm_eval_freepath", "cm_server_create", "cm_server_tune", "cm_server_destroy", "cm_job_submit",
    "cm_job_poll", "cm_job_wait", "cm_job_cancel", "cm_job_result", "cm_get_tuning", "cm_set_tuning", "cm_autotune",
)

JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = 0, 1, 2, 3, 4


class RunDesc(C.Structure):
    _fields_ = [("chamber", C.c_int), ("precision", C.c_int), ("npix", C.c_int), ("beam_width", C.c_double),
                ("pixel_center", C.POINTER(C.c_double)), ("pixel_energy", C.POINTER(C.c_double)),
                ("pixel_nprim", C.POINTER(C.c_int)), ("pixel_nbins", C.POINTER(C.c_int)), ("seed", C.c_uint64),
                ("hist_stride", C.c_int), ("wave", C.c_int), ("max_iterations", C.c_int),
                ("pixel_key", C.POINTER(C.c_uint64)), ("profile", C.c_int),
                ("elevation", C.POINTER(C.c_uint32)), ("azimuth", C.POINTER(C.c_uint32)),
                ("escape_log", C.c_void_p), ("escape_log_cap", C.c_int64),
                ("pixel_first", C.POINTER(C.c_int64))]


ELEVATION_COUNTS, AZIMUTH_COUNTS = 182, 362
# cm_escape_record
ESCAPE_RECORD = np.dtype([("electron", np.uint64), ("pixel", np.int32), ("step", np.int32), ("energy_eV", np.float64),
                          ("position", np.float64, 3), ("theta", np.float64), ("phi", np.float64)])


class Tuning(C.Structure):
    _fields_ = [("wave", C.c_int), ("tail_below", C.c_int), ("tail_steps", C.c_int), ("blocks_per_sm", C.c_int),
                ("ms", C.c_double), ("pool", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class JobInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("error", C.c_int), ("submit_s", C.c_double), ("start_s", C.c_double),
                ("end_s", C.c_double), ("primaries", C.c_int64), ("steps", C.c_int64)]


class RunStats(C.Structure):
    _fields_ = [("primaries", C.c_int64), ("steps", C.c_int64), ("scatter_events", C.c_int64),
                ("barrier_events", C.c_int64), ("escapes", C.c_int64), ("secondaries", C.c_int64),
                ("iterations", C.c_int64), ("device_ms", C.c_double), ("kernel_ms", C.c_double * 6),
                ("kernel_launches", C.c_int64 * 6), ("units", C.c_int64 * 4), ("step_launches", C.c_int64),
                ("step_units", C.c_int64), ("step_ms", C.c_double), ("ended_zero_energy", C.c_int64),
                ("ended_step_limit", C.c_int64), ("pool_restarts", C.c_int64)]

    KERNELS = ("flight", "elastic", "inelastic", "misc", "spawn", "tail")

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_[:8]}
        d["kernel_ms"] = dict(zip(self.KERNELS, list(self.kernel_ms)))
        d["kernel_launches"] = dict(zip(self.KERNELS, list(self.kernel_launches)))
        d["units"] = dict(zip(self.KERNELS[:4], list(self.units)))
        d["step_launches"] = self.step_launches
        d["step_units"] = self.step_units
        d["step_ms"] = self.step_ms
        d["ended_zero_energy"] = self.ended_zero_energy
        d["ended_step_limit"] = self.ended_step_limit
        d["pool_restarts"] = self.pool_restarts
        return d


class CMError(RuntimeError):
    """A CM_E* status from the library; .code is the status."""

    def __init__(self, msg, code=0):
        super().__init__(msg)
        self.code = code


_libs = {}


def load(path=LIBPATH):
    """Load the in-tree library (raises if it was not built)."""
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise CMError("libcudamonsel_b200.so not built; run `python -m cudamonsel_b200.build`")
    L = C.CDLL(path)
    d = C.POINTER(C.c_double)
    i = C.POINTER(C.c_int)
    ctx = C.c_void_p
    sig = {
        "cm_context_create": [C.c_int, C.POINTER(C.c_void_p)],
        "cm_context_destroy": [ctx],
        "cm_context_reset": [ctx],
        "cm_set_options": [ctx, C.c_int],
        "cm_get_tuning": [ctx, C.c_int, C.POINTER(Tuning)],
        "cm_set_tuning": [ctx, C.c_int, C.POINTER(Tuning)],
        "cm_autotune": [ctx, C.POINTER(RunDesc), C.POINTER(Tuning)],
        "cm_add_mott_element": [ctx, C.c_int, d, d],
        "cm_add_table": [ctx, C.c_int, i, d, d, i],
        "cm_add_material": [ctx, C.c_int, i, d, d, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, d, i],
        "cm_add_msm": [ctx, C.c_int, i],
        "cm_msm_add_nistmott": [ctx, C.c_int, C.c_int, i],
        "cm_msm_add_tabulated": [ctx, C.c_int, C.c_int, C.c_double, i, i],
        "cm_msm_add_fitted": [ctx, C.c_int, C.c_double, C.c_double, i],
        "cm_msm_add_phonon": [ctx, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, i],
        "cm_msm_add_polaron": [ctx, C.c_int, C.c_double, C.c_double, i],
        "cm_msm_set_csd_jln": [ctx, C.c_int, C.c_double],
        "cm_msm_set_min_e": [ctx, C.c_int, C.c_double],
        "cm_msm_set_barrier": [ctx, C.c_int, C.c_int, C.c_double],
        "cm_shape_sphere": [ctx, d, C.c_double, i],
        "cm_shape_planes": [ctx, C.c_int, d, d, i],
        "cm_shape_intersection": [ctx, C.c_int, C.c_int, i],
        "cm_shape_translate": [ctx, C.c_int, d],
        "cm_shape_rotate": [ctx, C.c_int, d, C.c_double, C.c_double, C.c_double],
        "cm_shape_union": [ctx, C.c_int, C.c_int, i],
        "cm_shape_cylinder": [ctx, d, d, C.c_double, i],
        "cm_shape_line": [ctx] + [C.c_double] * 7 + [i],
        "cm_region_add": [ctx, C.c_int, C.c_int, C.c_int, i],
        "cm_run": [ctx, C.POINTER(RunDesc), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(RunStats)],
        "cm_run_device": [ctx, C.POINTER(RunDesc), C.c_void_p, C.c_void_p, C.POINTER(RunStats), C.c_void_p],
        "cm_run_noalloc": [ctx, C.POINTER(RunDesc), C.c_void_p, C.c_void_p, C.POINTER(RunStats), C.c_void_p],
        "cm_server_create": [C.c_int, C.c_int, C.c_double, C.POINTER(C.c_void_p)],
        "cm_server_tune": [C.c_void_p, C.c_int, C.POINTER(Tuning)],
        "cm_server_destroy": [C.c_void_p],
        "cm_job_submit": [C.c_void_p, ctx, C.POINTER(RunDesc), i],
        "cm_job_poll": [C.c_void_p, C.c_int, C.POINTER(JobInfo)],
        "cm_job_wait": [C.c_void_p, C.c_int, C.c_double, C.POINTER(JobInfo)],
        "cm_job_cancel": [C.c_void_p, C.c_int],
        "cm_job_result": [C.c_void_p, C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(RunStats)],
        "cm_eval_nistmott": [ctx, C.c_int, C.c_int, C.c_int, d, d, d, d, C.c_int],
        "cm_eval_table": [ctx, C.c_int, C.c_int, d, C.c_int, d, C.c_int],
        "cm_eval_locate": [ctx, C.c_int, C.c_int, d, C.c_int, i, C.c_int],
        "cm_eval_pick": [ctx, C.c_int, C.c_int, d, d, C.c_int],
        "cm_eval_tabulated": [ctx, C.c_int, C.c_int, C.c_int, d, d, C.c_int],
        "cm_eval_elastic": [ctx, C.c_int, C.c_int, C.c_int, d, d, C.c_int],
        "cm_eval_csd": [ctx, C.c_int, C.c_int, d, d, C.c_int],
        "cm_eval_phonon": [ctx, C.c_int, C.c_int, C.c_int, d, d, C.c_int],
        "cm_eval_shape": [ctx, C.c_int, C.c_int, d, d],
        "cm_eval_barrier": [ctx, C.c_int, C.c_int, C.c_int, d, d, C.c_int],
        "cm_eval_freepath": [ctx, C.c_int, C.c_int, d, d, C.c_int],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.cm_last_error.restype = C.c_char_p
    L.cm_last_error.argtypes = []
    L.cm_version.restype = C.c_int
    _libs[path] = L
    return L


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(C.POINTER(C.c_int))


class Engine:
    """One cm_context on one CUDA device.  Methods mirror the C ABI (SI units)."""

    def __init__(self, device=0):
        self.L = load()
        h = C.c_void_p()
        self._check(self.L.cm_context_create(device, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.cm_context_destroy(self.h)
            self.h = None

    def reset(self):
        """Forget the scene so this context can describe another (cm_context_reset)."""
        self._check(self.L.cm_context_reset(self.h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise CMError("cudamonsel_b200 error %d: %s" % (rc, self.L.cm_last_error().decode()), rc)

    def _out(self, fn, *args):
        o = C.c_int(-1)
        self._check(fn(self.h, *args, C.byref(o)))
        return o.value

    # ---- scene (same method names as oracle/pyoracle.Scene via scene.SceneSpec)
    def set_options(self, opt):
        self._check(self.L.cm_set_options(self.h, opt))

    def tuning(self, precision=PREC_FP64):
        t = Tuning()
        self._check(self.L.cm_get_tuning(self.h, precision, C.byref(t)))
        return t

    def set_tuning(self, precision=PREC_FP64, wave=0, tail_below=0, tail_steps=0, blocks_per_sm=0, pool=0):
        t = Tuning(wave, tail_below, tail_steps, blocks_per_sm, 0.0, pool)
        self._check(self.L.cm_set_tuning(self.h, precision, C.byref(t)))

    def autotune(self, chamber, centers, energies, nprim, nbins, beam_width, seed, precision=PREC_FP64,
                 pixel_keys=None):
        """cm_autotune on this workload (host arrays); returns the Tuning kept for later runs."""
        desc, keep, _, _ = _run_desc(chamber, centers, energies, nprim, nbins, beam_width, seed, precision, pixel_keys)
        t = Tuning()
        self._check(self.L.cm_autotune(self.h, C.byref(desc), C.byref(t)))
        return t

    def mott(self, Z, spwem, x1):
        a, pa = _d(spwem)
        b, pb = _d(x1)
        self._check(self.L.cm_add_mott_element(self.h, Z, pa, pb))

    def table(self, dim, n, axes, values):
        ni, pn = _i(n)
        ax, pax = _d(np.concatenate([np.asarray(a, dtype=np.float64) for a in axes]))
        v, pv = _d(np.asarray(values, dtype=np.float64).ravel())
        return self._out(self.L.cm_add_table, dim, pn, pax, pv)

    def material(self, Z, A, wf, density, workfunction, ecb, bandgap, core=()):
        z, pz = _i(Z if len(Z) else [0])
        a, pa = _d(A if len(A) else [0])
        w, pw = _d(wf if len(wf) else [0])
        c, pc = _d(core if len(core) else [0])
        return self._out(self.L.cm_add_material, len(Z), pz, pa, pw, density, workfunction, ecb, bandgap, len(core), pc)

    def msm(self, material):
        return self._out(self.L.cm_add_msm, material)

    def nistmott(self, msm, method=1):
        return self._out(self.L.cm_msm_add_nistmott, msm, method)

    def tabulated(self, msm, method_se, offset, tables):
        t, pt = _i(tables)
        return self._out(self.L.cm_msm_add_tabulated, msm, method_se, offset, pt)

    def fitted(self, msm, energy_se_gen, break_e):
        return self._out(self.L.cm_msm_add_fitted, msm, energy_se_gen, break_e)

    def phonon(self, msm, ratemult, phonon_e, temperature, eps0, eps_inf):
        return self._out(self.L.cm_msm_add_phonon, msm, ratemult, phonon_e, temperature, eps0, eps_inf)

    def polaron(self, msm, prefactor, extinction):
        return self._out(self.L.cm_msm_add_polaron, msm, prefactor, extinction)

    def csd_jln(self, msm, break_e):
        self._check(self.L.cm_msm_set_csd_jln(self.h, msm, break_e))

    def min_e(self, msm, e):
        self._check(self.L.cm_msm_set_min_e(self.h, msm, e))

    def barrier(self, msm, classical, lam):
        self._check(self.L.cm_msm_set_barrier(self.h, msm, classical, lam))

    def sphere(self, c, r):
        a, pa = _d(c)
        return self._out(self.L.cm_shape_sphere, pa, r)

    def planes(self, normals, points):
        n, pn = _d(normals)
        p, pp = _d(points)
        return self._out(self.L.cm_shape_planes, len(n) // 3, pn, pp)

    def intersection(self, a, b):
        return self._out(self.L.cm_shape_intersection, a, b)

    def translate(self, shape, d):
        a, pa = _d(d)
        self._check(self.L.cm_shape_translate(self.h, shape, pa))

    def rotate(self, shape, pivot, phi, theta, psi):
        a, pa = _d(pivot)
        self._check(self.L.cm_shape_rotate(self.h, shape, pa, phi, theta, psi))

    def union(self, a, b):
        return self._out(self.L.cm_shape_union, a, b)

    def cylinder(self, end0, end1, radius):
        a, pa = _d(end0)
        b, pb = _d(end1)
        return self._out(self.L.cm_shape_cylinder, pa, pb, radius)

    def line(self, topz, width, length, thetal, thetar, radl=0.0, radr=0.0):
        return self._out(self.L.cm_shape_line, topz, width, length, thetal, thetar, radl, radr)

    def region(self, parent, msm, shape):
        return self._out(self.L.cm_region_add, parent, msm, shape)

    # ---- runs
    def run(self, chamber, centers, energies, nprim, nbins, beam_width, seed, precision=PREC_FP64, wave=0,
            max_iterations=0, pixel_keys=None, profile=0, angles=False, escape_log_cap=0, first_primary=None):
        """cm_run: (back, fwd, stats); with angles or an escape log also a dict of BackscatterStats'
        elevation [npix, 182] and azimuthal [npix, 362] histograms and the escape records.  first_primary
        (per pixel, or None: 0) is the index of each pixel's first primary, for a scan run in parts."""
        centers = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
        npix = len(centers)
        e, pe = _d(np.broadcast_to(np.asarray(energies, dtype=np.float64), (npix,)).copy())
        c, pc = _d(centers.ravel())
        n, pn = _i(np.broadcast_to(np.asarray(nprim), (npix,)).copy())
        b, pb = _i(np.broadcast_to(np.asarray(nbins), (npix,)).copy())
        stride = int(b.max()) + 2
        keys = None
        if pixel_keys is not None:
            keys = np.ascontiguousarray(pixel_keys, dtype=np.uint64)
        desc = RunDesc(chamber, precision, npix, beam_width, pc, pe, pn, pb, seed, stride, wave, max_iterations,
                       keys.ctypes.data_as(C.POINTER(C.c_uint64)) if keys is not None else None, profile)
        first = None
        if first_primary is not None:
            first = np.ascontiguousarray(np.broadcast_to(np.asarray(first_primary), (npix,)), dtype=np.int64)
            desc.pixel_first = first.ctypes.data_as(C.POINTER(C.c_int64))
        extra = None
        if angles or escape_log_cap:
            extra = {}
            if angles:
                extra["elevation"] = np.zeros((npix, ELEVATION_COUNTS), dtype=np.uint32)
                extra["azimuth"] = np.zeros((npix, AZIMUTH_COUNTS), dtype=np.uint32)
                desc.elevation = extra["elevation"].ctypes.data_as(C.POINTER(C.c_uint32))
                desc.azimuth = extra["azimuth"].ctypes.data_as(C.POINTER(C.c_uint32))
            if escape_log_cap:
                log = np.zeros(int(escape_log_cap), dtype=ESCAPE_RECORD)
                desc.escape_log = log.ctypes.data
                desc.escape_log_cap = int(escape_log_cap)
        back = np.zeros((npix, stride), dtype=np.uint32)
        fwd = np.zeros((npix, stride), dtype=np.uint32)
        st = RunStats()
        self._check(self.L.cm_run(self.h, C.byref(desc), back.ctypes.data_as(C.POINTER(C.c_uint32)),
                                  fwd.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(st)))
        if extra is None:
            return back, fwd, st
        if escape_log_cap:
            extra["escape_log"] = log[:min(int(escape_log_cap), int(st.escapes))]
        return back, fwd, st, extra

    def run_device(self, desc, back_ptr, fwd_ptr, stream_ptr=None):
        st = RunStats()
        self._check(self.L.cm_run_device(self.h, C.byref(desc), C.c_void_p(back_ptr), C.c_void_p(fwd_ptr),
                                         C.byref(st), C.c_void_p(stream_ptr) if stream_ptr else None))
        return st

    def run_noalloc(self, desc, back_ptr, fwd_ptr, stream_ptr=None):
        """cm_run_device without device allocations (fixed scratch array; see the header)."""
        st = RunStats()
        self._check(self.L.cm_run_noalloc(self.h, C.byref(desc), C.c_void_p(back_ptr), C.c_void_p(fwd_ptr),
                                          C.byref(st), C.c_void_p(stream_ptr) if stream_ptr else None))
        return st

    # ---- per-function entry points
    def eval_nistmott(self, Z, E, u, precision=PREC_FP64, method=1):
        E, pE = _d(E)
        u, pu = _d(u)
        s = np.zeros(len(E))
        t = np.zeros(len(E))
        self._check(self.L.cm_eval_nistmott(self.h, Z, method, len(E), pE, pu, s.ctypes.data_as(C.POINTER(C.c_double)),
                                            t.ctypes.data_as(C.POINTER(C.c_double)), precision))
        return s, t

    def _eval(self, fn, args, inp, n_out, precision=None):
        inp = np.ascontiguousarray(inp, dtype=np.float64)
        n = inp.shape[0]
        out = np.zeros((n, n_out), dtype=np.float64)
        extra = () if precision is None else (precision,)
        self._check(fn(self.h, *args, n, inp.ctypes.data_as(C.POINTER(C.c_double)),
                       out.ctypes.data_as(C.POINTER(C.c_double)), *extra))
        return out

    def eval_table(self, table, x3, order, precision=PREC_FP64):
        x3 = np.ascontiguousarray(x3, dtype=np.float64)
        out = np.zeros(len(x3))
        self._check(self.L.cm_eval_table(self.h, table, len(x3), x3.ctypes.data_as(C.POINTER(C.c_double)), order,
                                         out.ctypes.data_as(C.POINTER(C.c_double)), precision))
        return out

    def eval_locate(self, table, x3, order, precision=PREC_FP64):
        """cm_eval_locate: int array [n, 6] of (first, nearest) per axis (-1 for missing axes)."""
        x3 = np.ascontiguousarray(x3, dtype=np.float64)
        out = np.zeros((len(x3), 6), dtype=np.int32)
        self._check(self.L.cm_eval_locate(self.h, table, len(x3), x3.ctypes.data_as(C.POINTER(C.c_double)), order,
                                          out.ctypes.data_as(C.POINTER(C.c_int)), precision))
        return out

    def eval_pick(self, msm, inp, precision=PREC_FP64):
        """cm_eval_pick: [n, 2] of (mechanism index, total rate in 1/m) for rows (E in J, deviate)."""
        return self._eval(self.L.cm_eval_pick, (msm,), inp, 2, precision)

    def eval_tabulated(self, msm, mech, inp, precision=PREC_FP64):
        return self._eval(self.L.cm_eval_tabulated, (msm, mech), inp, 12, precision)

    def eval_elastic(self, msm, mech, inp, precision=PREC_FP64):
        return self._eval(self.L.cm_eval_elastic, (msm, mech), inp, 6, precision)

    def eval_csd(self, msm, inp, precision=PREC_FP64):
        return self._eval(self.L.cm_eval_csd, (msm,), inp, 3, precision)

    def eval_phonon(self, msm, mech, inp, precision=PREC_FP64):
        return self._eval(self.L.cm_eval_phonon, (msm, mech), inp, 6, precision)

    def eval_shape(self, shape, p01):
        return self._eval(self.L.cm_eval_shape, (shape,), p01, 6)

    def eval_barrier(self, frm, to, inp, precision=PREC_FP64):
        return self._eval(self.L.cm_eval_barrier, (frm, to), inp, 8, precision)

    def eval_freepath(self, msm, inp, precision=PREC_FP64):
        return self._eval(self.L.cm_eval_freepath, (msm,), inp, 1, precision)[:, 0]


def _run_desc(chamber, centers, energies, nprim, nbins, beam_width, seed, precision, pixel_keys=None, wave=0,
              max_iterations=0, profile=0):
    """A RunDesc over host arrays, and the arrays it points at (keep them alive while it is used)."""
    centers = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
    npix = len(centers)
    e, pe = _d(np.broadcast_to(np.asarray(energies, dtype=np.float64), (npix,)).copy())
    c, pc = _d(centers.ravel())
    n, pn = _i(np.broadcast_to(np.asarray(nprim), (npix,)).copy())
    b, pb = _i(np.broadcast_to(np.asarray(nbins), (npix,)).copy())
    stride = int(b.max()) + 2
    keys = None if pixel_keys is None else np.ascontiguousarray(pixel_keys, dtype=np.uint64)
    desc = RunDesc(chamber, precision, npix, beam_width, pc, pe, pn, pb, seed, stride, wave, max_iterations,
                   keys.ctypes.data_as(C.POINTER(C.c_uint64)) if keys is not None else None, profile)
    return desc, (c, e, n, b, keys), npix, stride


class Server:
    """cm_server: a continuously batching job server on one GPU; up to `slots` jobs share a batch."""

    def __init__(self, device=0, slots=4, budget_gb=16.0):
        self.L = load()
        h = C.c_void_p()
        rc = self.L.cm_server_create(device, slots, budget_gb, C.byref(h))
        if rc:
            raise CMError("cudamonsel_b200 error %d: %s" % (rc, self.L.cm_last_error().decode()), rc)
        self.h = h
        self.shape = {}

    def _check(self, rc):
        if rc != 0:
            raise CMError("cudamonsel_b200 error %d: %s" % (rc, self.L.cm_last_error().decode()), rc)

    def close(self):
        if getattr(self, "h", None):
            self.L.cm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, engine, chamber, centers, energies, nprim, nbins, beam_width, seed, precision=PREC_FP32,
               pixel_keys=None):
        """Queue a job: the scene held by `engine` (copied now) and host pixel arrays (copied now)."""
        desc, keep, npix, stride = _run_desc(chamber, centers, energies, nprim, nbins, beam_width, seed, precision,
                                             pixel_keys)
        job = C.c_int(-1)
        self._check(self.L.cm_job_submit(self.h, engine.h, C.byref(desc), C.byref(job)))
        self.shape[job.value] = (npix, stride)
        return job.value

    def tune(self, precision, wave=0, tail_below=0, tail_steps=0, blocks_per_sm=0, pool=0):
        """Launch settings of the batches of one precision that start after the call (0 = default)."""
        t = Tuning(wave, tail_below, tail_steps, blocks_per_sm, 0.0, pool)
        self._check(self.L.cm_server_tune(self.h, precision, C.byref(t)))

    def poll(self, job):
        info = JobInfo()
        self._check(self.L.cm_job_poll(self.h, job, C.byref(info)))
        return info

    def wait(self, job, timeout=-1.0):
        info = JobInfo()
        self._check(self.L.cm_job_wait(self.h, job, timeout, C.byref(info)))
        return info

    def cancel(self, job):
        self._check(self.L.cm_job_cancel(self.h, job))

    def result(self, job):
        """Tallies (back, fwd as [npix, stride]) and RunStats of a finished job; the server then forgets it."""
        npix, stride = self.shape.pop(job)
        back = np.zeros((npix, stride), dtype=np.uint32)
        fwd = np.zeros((npix, stride), dtype=np.uint32)
        st = RunStats()
        self._check(self.L.cm_job_result(self.h, job, back.ctypes.data_as(C.POINTER(C.c_uint32)),
                                         fwd.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(st)))
        return back, fwd, st
