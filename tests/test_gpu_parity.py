"""Per-function parity of the CUDA kernels with the reference, through the C ABI.

Inputs are the golden vectors dumped from the reference (tests/golden/) with
their injected uniform deviates; the expected outputs are the reference's own
(which the C oracle reproduces bit for bit, tests/test_oracle_golden.py).

Tolerances, written per check:
  FP64 kernels: values within 1e-9 relative (the engine computes in eV/nm, the
    reference in J/m, so results differ by a few ulp), table-window and
    mechanism/element selections identical;
  FP32 kernels: cross sections, rates, table values, sampled angles, energy
    losses and SE energies within 1e-6 relative; directions within 1e-6
    (inelastic) and 5e-6 (elastic) absolute; every bound on the largest error, not a quantile;
    selections identical (an element pick whose deviate lies within float rounding of a cumulative
    cross section is counted and excluded, and none differs).
The reference's 3-D theta interpolation extrapolates from the first four
energy nodes (NULagrangeInterpolation.cu:236); its result amplifies rounding
by up to (E/E3)^3, so directions after such events are compared only where
the sampled theta stays below 10 rad (in FP64) and statistically otherwise.

FP32 kernels see float inputs: an energy of 19999.99999 eV arrives as
20000.0f and legitimately takes the other branch.  FP32 checks therefore
compare against the oracle evaluated on the float-rounded inputs.
"""
import numpy as np
import pytest

from conftest import EV, golden, golden_lines

pytestmark = pytest.mark.gpu

FP64, FP32 = 0, 1


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def unit(theta, phi):
    return np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)], axis=1)


@pytest.fixture(scope="module")
def lines_engine(engine):
    from cudamonsel_b200 import scenes
    sc = scenes.lines()
    h = scenes.build_engine(sc, engine)
    return engine, h


FROMSI = 1.0 / 1.60217653e-19


def f32_energy(E):
    """The SI energy whose eV value is exactly the float the FP32 kernels compute with."""
    return np.float32(np.asarray(E) * FROMSI).astype(np.float64) / FROMSI


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def oracle_nistmott(b, Z, E, u):
    import ctypes as C
    import pyoracle as po
    n = len(E)
    s, t = np.zeros(n), np.zeros(n)
    nd = np.zeros(n, dtype=np.int32)
    b.L.cmo_eval_nistmott(b.h, Z, n, po.dp(np.ascontiguousarray(E)), po.dp(np.ascontiguousarray(u)),
                          s.ctypes.data_as(C.POINTER(C.c_double)), t.ctypes.data_as(C.POINTER(C.c_double)),
                          nd.ctypes.data_as(C.POINTER(C.c_int)))
    return s, t


@pytest.mark.parametrize("Z", [1, 6, 8, 14])
def test_nistmott_fp64(lines_engine, Z):
    """NISTMottRS cross section and sampled angle (JMONSEL/NISTMottRS.cu:103-154), FP64 vs the reference."""
    e, h = lines_engine
    g = golden("nistmott")
    rows = g[g[:, 0] == Z]
    sig, th = e.eval_nistmott(Z, rows[:, 1], np.ascontiguousarray(rows[:, 2:4]), FP64)
    r = rel(sig, rows[:, 4])
    print("Z=%d FP64 sigma max rel %.3g" % (Z, r.max()))
    assert r.max() < 1e-9
    d = np.abs(th - rows[:, 5])
    for i in np.argsort(-d)[:4]:
        print("  E %.17g eV u %.17g %.17g theta %.17g ref %.17g" % (rows[i, 1] * FROMSI, rows[i, 2], rows[i, 3], th[i],
                                                                    rows[i, 5]))
    print("Z=%d FP64 theta max abs %.3g, cases above 1e-9: %d" % (Z, d.max(), (d > 1e-9).sum()))
    assert d.max() < 1e-9


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("method", [2, 3])
def test_nistmott_methods_2_3(lines_engine, oracle_lines, method, prec):
    """NISTMottRS methods 2 and 3 (extrapolation below 100 eV, JMONSEL/NISTMottRS.cu:76-119): FP64 against the
    reference's golden vectors, FP32 against the oracle on float-rounded energies and deviates."""
    import ctypes as C
    import pyoracle as po
    e, h = lines_engine
    b, _, _ = oracle_lines
    g = golden("nistmott23")
    for Z in (1, 6, 8, 14):
        rows = g[(g[:, 0] == method) & (g[:, 1] == Z)]
        n = len(rows)
        if prec == FP64:
            E, u = rows[:, 2], np.ascontiguousarray(rows[:, 3:5])
            rs, rt = rows[:, 5], rows[:, 6]
        else:
            E, u = f32_energy(rows[:, 2]), np.ascontiguousarray(f32(rows[:, 3:5]))
            rs, rt = np.zeros(n), np.zeros(n)
            nd = np.zeros(n, dtype=np.int32)
            b.L.cmo_eval_nistmott_method(b.h, Z, method, n, po.dp(np.ascontiguousarray(E)), po.dp(u),
                                         rs.ctypes.data_as(C.POINTER(C.c_double)),
                                         rt.ctypes.data_as(C.POINTER(C.c_double)), nd.ctypes.data_as(C.POINTER(C.c_int)))
        sig, th = e.eval_nistmott(Z, np.ascontiguousarray(E), u, prec, method)
        tol = 1e-9 if prec == FP64 else 1e-6
        r = rel(sig, rs)
        d = np.abs(th - rt) / np.maximum(rt, 1e-6) if prec == FP32 else np.abs(th - rt)
        print("method %d Z=%d sigma max rel %.3g theta max %.3g" % (method, Z, r.max(), d.max()))
        assert r.max() < tol and d.max() < tol


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_browning_with_fixes(prec):
    """Browning's cross section and screened angle below the NIST Mott range as JMONSEL computes them
    (BrowningEmpiricalCrossSection.cu:24-45 with the element's Z; CM_OPT_JMONSEL_FIXES), where the compiled
    reference reads Z through a dangling reference and always takes the isotropic branch: engine vs the
    oracle in its fixes mode on 2-49 eV and uniform deviates, FP32 on float-rounded inputs."""
    import pyoracle
    from cudamonsel_b200 import capi, scenes
    sc = scenes.lines()
    sc.spec.options = 1
    e = capi.Engine(0)
    scenes.build_engine(sc, e)
    b, _ = pyoracle.build_oracle(sc)
    rng = np.random.default_rng(17)
    n = 4000
    E = np.exp(rng.uniform(np.log(2.0), np.log(49.0), n)) / FROMSI
    u = rng.random((n, 2))
    if prec == FP32:
        E, u = f32_energy(E), f32(u)
    u = np.ascontiguousarray(u)
    for Z in (1, 6, 8, 14):
        sig, th = e.eval_nistmott(Z, np.ascontiguousarray(E), u, prec)
        rs, rt = oracle_nistmott(b, Z, E, u)
        r = rel(sig, rs)
        d = np.abs(th - rt) if prec == FP64 else np.abs(th - rt) / np.maximum(rt, 1e-6)
        iso = np.abs(np.cos(rt) - (1 - 2 * u[:, 1])) < 1e-12
        print("Z=%d prec %d sigma max rel %.3g theta max %.3g (screened branch in %d of %d)" % (
            Z, prec, r.max(), d.max(), (~iso).sum(), n))
        assert (~iso).sum() > n // 10  # the screened branch is taken, not only the isotropic one
        assert r.max() < (1e-9 if prec == FP64 else 1e-6)
        assert d.max() < (1e-9 if prec == FP64 else 1e-6)
    e.close()


def test_nistmott_sweep(lines_engine, oracle_lines):
    """Sampled Mott angle over a fine grid of deviates and energies (FP64 vs the oracle)."""
    e, h = lines_engine
    b, _, _ = oracle_lines
    for Z in (1, 14):
        for EeV in (60.0, 461.16647528186616, 5854.963):
            u1 = np.linspace(0.0005, 0.9995, 1000)
            E = np.full(len(u1), EeV / FROMSI)
            u = np.ascontiguousarray(np.column_stack([u1, np.full(len(u1), 0.5)]))
            s, th = e.eval_nistmott(Z, E, u, FP64)
            rs, rt = oracle_nistmott(b, Z, E, u)
            bad = np.abs(th - rt) > 1e-9
            if bad.any():
                idx = np.where(bad)[0]
                print("Z=%d E=%g: %d bad, u from %.4f to %.4f; first %s" % (Z, EeV, bad.sum(), u1[idx[0]], u1[idx[-1]],
                      [(round(u1[i], 4), round(th[i], 6), round(rt[i], 6)) for i in idx[:6]]))
            assert not bad.any()


@pytest.mark.parametrize("Z", [1, 6, 8, 14])
def test_nistmott_fp32(lines_engine, oracle_lines, Z):
    """FP32 NISTMottRS vs the oracle on float-rounded energies and deviates."""
    e, h = lines_engine
    b, _, _ = oracle_lines
    g = golden("nistmott")
    rows = g[g[:, 0] == Z]
    E = f32_energy(rows[:, 1])
    u = np.ascontiguousarray(f32(rows[:, 2:4]))
    sig, th = e.eval_nistmott(Z, E, u, FP32)
    rs, rt = oracle_nistmott(b, Z, E, u)
    r = rel(sig, rs)
    print("Z=%d FP32 sigma max rel %.3g" % (Z, r.max()))
    assert r.max() < 1e-6
    d = np.abs(th - rt) / np.maximum(rt, 1e-6)
    print("Z=%d FP32 theta max rel %.3g, median %.3g" % (Z, d.max(), np.median(d)))
    for k in np.argsort(d)[-3:]:
        print("  E %.6g eV u %.6g %.6g theta %.9g ref %.9g" % (E[k] / EV, u[k, 0], u[k, 1], th[k], rt[k]))
    assert d.max() < 1e-6


def oracle_eval(b, fn, args, inp, nout):
    import ctypes as C
    import pyoracle as po
    inp = np.ascontiguousarray(inp, dtype=np.float64)
    out = np.zeros((len(inp), nout))
    getattr(b.L, fn)(b.h, *args, len(inp), po.dp(inp), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def theta_window(b, x0):
    """Window start NULagrangeInterpolation::locate picks on the theta table's energy axis
    (0: no extrapolation by the reference's d3 quirk)."""
    return np.array([b.L.cmo_table_window(b.h, 2, float(x)) for x in x0])


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_tables(lines_engine, oracle_lines, prec):
    """NUTableInterpolation on the four Si tables (engine converts axes and values to eV/nm)."""
    import ctypes as C
    import pyoracle as po
    e, h = lines_engine
    b, ho, _ = oracle_lines
    g = golden("nutable")
    for t in range(4):
        rows = g[g[:, 0] == t]
        order = int(rows[0, 4])
        x = np.ascontiguousarray(rows[:, 1:4])
        if prec == FP32:
            x = np.column_stack([f32_energy(x[:, 0]), f32(x[:, 1]), f32(x[:, 2])])
            ref = np.zeros(len(x))
            b.L.cmo_eval_table(b.h, t, len(x), po.dp(x), order, ref.ctypes.data_as(C.POINTER(C.c_double)))
        else:
            ref = rows[:, 5]
        out = e.eval_table(t, x, order, prec)
        r = rel(out, ref)
        if t == 2:
            # beyond the first energy window the reference extrapolates (d3 quirk) and amplifies the
            # rounding of its inputs by the Lebesgue constant of the first four energy nodes at E; both
            # precisions evaluate the 3-D table in double, so the bound holds there too (as a maximum)
            first = theta_window(b, x[:, 0]) == 0
            print("table %d prec %d first-window max rel %.3g, extrapolated max rel %.3g over %d" % (
                t, prec, r[first].max(), r[~first].max(), (~first).sum()))
            assert first.sum() > 20 and (~first).sum() > 20
            assert r[first].max() < (1e-9 if prec == FP64 else 1e-6)
            assert r[~first].max() < 1e-6
        else:
            print("table %d prec %d max rel %.3g" % (t, prec, r.max()))
            assert r.max() < (1e-9 if prec == FP64 else 1e-6)


def tabulated_inputs_and_ref(rows, prec, b, ho):
    inp = np.ascontiguousarray(rows[:, 0:9])
    if prec == FP32:
        inp = np.column_stack([f32_energy(inp[:, 0]), f32(inp[:, 1:9])])
    import ctypes as C
    import pyoracle as po
    ref = np.zeros((len(inp), 10))
    b.L.cmo_eval_tabulated_stride(b.h, ho["si"], 1, len(inp), po.dp(inp), ref.ctypes.data_as(C.POINTER(C.c_double)), 10)
    if prec == FP64:
        assert (ref[:, :9] == rows[:, 9:18]).all()  # the oracle is the reference on these inputs
    return inp, ref


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_tabulated_inelastic(lines_engine, oracle_lines, prec):
    """TabulatedInelasticSM scatter: energy loss, SE energy and generation branch, deviates used.
    Outcomes downstream of the sampled theta (Eq, the SE branch, its energy and direction) are
    compared where theta comes from the first energy window of the table; beyond it the reference's
    d3 extrapolation amplifies rounding and only the energy loss and rate are compared."""
    e, h = lines_engine
    b, ho, _ = oracle_lines
    rows = golden("tabinel")
    inp, ref = tabulated_inputs_and_ref(rows, prec, b, ho)
    out = e.eval_tabulated(h["si"], 1, inp, prec)
    first = theta_window(b, inp[:, 0] + scenes_eV(13.54)) == 0
    print("cases %d, first-window %d" % (len(inp), first.sum()))
    tol = 1e-9 if prec == FP64 else 1e-6
    r = rel(out[:, 0], ref[:, 0])
    print("prec %d rate max rel %.3g" % (prec, r.max()))
    assert r.max() < tol
    same_se = out[:, 5] == ref[:, 4]
    same_dev = out[:, 10] == ref[:, 8]
    print("SE decision agreement %.5f (first window %.5f), deviate count agreement %.5f (first window %.5f)" % (
        same_se.mean(), same_se[first].mean(), same_dev.mean(), same_dev[first].mean()))
    for i in np.where(~(same_se & same_dev))[0][:10]:
        print("  decision differs: E %.9g eV theta %.9g phi %.9g u %s: engine SE %d deviates %d, oracle %d %d" % (
            inp[i, 0] * FROMSI, inp[i, 1], inp[i, 2], np.array2string(inp[i, 3:9], precision=9), out[i, 5], out[i, 10],
            ref[i, 4], ref[i, 8]))
    assert same_se.all() and same_dev.all()
    ok = same_se & same_dev
    dE0 = inp[:, 0] - ref[:, 1]
    dE1 = inp[:, 0] - out[:, 1]
    if prec == FP64:
        r = (np.abs(dE1 - dE0) / np.maximum(np.abs(dE0), 1e-22))[ok]
        print("energy loss max rel %.3g" % r.max())
        assert r.max() < 1e-9
    else:
        # in FP32 the loss is read off the float energy E' = E - dE, whose rounding is up to half a
        # float spacing of E: the bound is 1e-6 of the loss plus one spacing of E
        spacing = np.spacing(np.float32(inp[:, 0] * FROMSI)).astype(np.float64) / FROMSI
        q = (np.abs(dE1 - dE0) / (1e-6 * np.abs(dE0) + spacing))[ok]
        print("energy loss error / bound: max %.3g, 99.9%% %.3g" % (q.max(), np.quantile(q, 0.999)))
        assert q.max() < 1.0
    th = rel(out[first, 11], ref[first, 9])
    print("theta (first window) max rel %.3g" % th.max())
    assert th.max() < (1e-9 if prec == FP64 else 1e-6)
    se = ok & first & (ref[:, 4] == 1)
    r = rel(out[se, 6], ref[se, 5])
    print("SE energy max rel %.3g over %d" % (r.max(), se.sum()))
    assert r.max() < (1e-9 if prec == FP64 else 1e-6)
    tame = ok & first
    err = np.abs(out[:, 2:5] - unit(ref[:, 2], ref[:, 3])).max(axis=1)
    print("PE direction max abs err (first window) %.3g over %d" % (err[tame].max(), tame.sum()))
    assert err[tame].max() < (1e-7 if prec == FP64 else 1e-6)
    serr = np.abs(out[:, 7:10] - unit(ref[:, 6], ref[:, 7])).max(axis=1)
    print("SE direction max abs err %.3g over %d" % (serr[se].max(), se.sum()))
    assert serr[se].max() < (1e-7 if prec == FP64 else 1e-6)


def scenes_eV(x):
    return x * EV


@pytest.mark.parametrize("prec", [FP64, FP32])
@pytest.mark.parametrize("mat", [0, 1])
def test_elastic(lines_engine, oracle_lines, mat, prec):
    """SelectableElasticSM: rate, element pick (PMMA: H, O, C), deflected direction."""
    e, h = lines_engine
    b, ho, _ = oracle_lines
    g = golden("elastic")
    rows = g[g[:, 0] == mat]
    msm, omsm = (h["si"], ho["si"]) if mat == 0 else (h["pmma"], ho["pmma"])
    inp = np.ascontiguousarray(rows[:, 1:8])
    if prec == FP64:
        ref = rows[:, 8:13]
    else:
        inp = np.column_stack([f32_energy(inp[:, 0]), f32(inp[:, 1:7])])
        ref = oracle_eval(b, "cmo_eval_elastic", (omsm, 0), inp, 5)
    out = e.eval_elastic(msm, 0, inp, prec)
    r = rel(out[:, 0], ref[:, 0])
    print("mat %d prec %d rate max rel %.3g" % (mat, prec, r.max()))
    assert r.max() < (1e-9 if prec == FP64 else 1e-6)
    sameZ = out[:, 4] == ref[:, 3]
    print("element agreement %.5f" % sameZ.mean())
    if prec == FP64:
        assert sameZ.all()
    else:
        # a float cannot resolve the pick where u * total lies within float rounding of a cumulative
        # cross section: those cases are where the oracle's own pick changes when u moves by 2e-6
        lo, hi = inp.copy(), inp.copy()
        lo[:, 3] *= 1 - 2e-6
        hi[:, 3] = np.minimum(hi[:, 3] * (1 + 2e-6), 1.0)
        edge = (oracle_eval(b, "cmo_eval_elastic", (omsm, 0), lo, 5)[:, 3] !=
                oracle_eval(b, "cmo_eval_elastic", (omsm, 0), hi, 5)[:, 3])
        for i in np.where(~sameZ)[0]:
            print("  element differs at E %.9g eV u %.9g (within rounding of a boundary: %s)" % (
                inp[i, 0] * FROMSI, inp[i, 3], bool(edge[i])))
        print("element picks within float rounding of a boundary: %d of %d" % (edge.sum(), len(edge)))
        assert sameZ[~edge].all()
    err = np.abs(out[:, 1:4] - unit(ref[:, 1], ref[:, 2])).max(axis=1)[sameZ]
    print("direction max abs err %.3g, 99.9%% %.3g" % (err.max(), np.quantile(err, 0.999)))
    assert err.max() < (1e-8 if prec == FP64 else 5e-6)
    assert (out[:, 5] == ref[:, 4]).all()


def window_inputs(axes):
    """Arguments on both sides of every abscissa and of every midpoint between neighbours, one and two
    float spacings away (in the units the FP32 kernels compute in: eV for energies), so that each one
    has a well-defined window and nearest node in both precisions."""
    xs = []
    for a in axes:
        pts = np.concatenate([a, 0.5 * (a[1:] + a[:-1])])
        f = pts.astype(np.float32)
        for k in (1, 2):
            up, dn = f.copy(), f.copy()
            for _ in range(k):
                up = np.nextafter(up, np.float32(np.inf))
                dn = np.nextafter(dn, np.float32(-np.inf))
            xs.append(np.concatenate([up, dn]).astype(np.float64))
    return xs


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_table_windows_are_exact(lines_engine, oracle_lines, prec):
    """NULagrangeInterpolation::locate (JMONSELutils/NULagrangeInterpolation.cu:5-68) on the four Si tables:
    the window start and nearest node of every axis, identical to the oracle (the reference's locate, pinned
    bit for bit) for the golden arguments and for arguments one and two float spacings either side of every
    abscissa and every midpoint (FP32: the float arguments the kernels see, compared on the double axes)."""
    import ctypes as C
    import pyoracle as po
    from cudamonsel_b200 import data
    e, h = lines_engine
    b, ho, _ = oracle_lines
    g = golden("nutable")
    tables = data.si_tables()
    total = 0
    for t in range(4):
        dim, n, axes, vals = data.read_nu_table(tables[t])
        ax = [np.asarray(axes[k]) for k in range(dim)]
        order = int(g[g[:, 0] == t][0, 4])
        rows = [g[g[:, 0] == t][:, 1:4]]
        ax_eV = [ax[0] * FROMSI] + ax[1:]  # energies in eV, where the FP32 arguments are floats
        per_axis = [window_inputs([a]) for a in ax_eV]
        for k in range(dim):
            for xk in per_axis[k]:
                x = np.zeros((len(xk), 3))
                for j in range(dim):  # the other axes at a fixed interior point
                    x[:, j] = ax_eV[j][len(ax_eV[j]) // 3]
                x[:, k] = xk
                x[:, 0] /= FROMSI  # the energy axis in J, as cm_eval_locate takes it
                rows.append(x)
        x = np.ascontiguousarray(np.concatenate(rows))
        if prec == FP32:
            x = np.column_stack([f32_energy(x[:, 0]), f32(x[:, 1]), f32(x[:, 2])])
        got = e.eval_locate(t, x, order, prec)
        want = np.zeros((len(x), 6), dtype=np.int32)
        b.L.cmo_table_locate(b.h, t, len(x), po.dp(x), order, want.ctypes.data_as(C.POINTER(C.c_int)))
        bad = np.where((got != want).any(axis=1))[0]
        for i in bad[:8]:
            print("  table %d x %s: engine %s oracle %s" % (t, x[i], got[i], want[i]))
        print("table %d prec %d: %d arguments, windows identical: %s" % (t, prec, len(x), len(bad) == 0))
        total += len(x)
        assert len(bad) == 0
    assert total > 2000


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("mat", ["si", "pmma"])
def test_mechanism_pick(lines_engine, oracle_lines, mat, prec):
    """MONSEL_MaterialScatterModel::scatter's choice of mechanism (MONSEL_MaterialScatterModel.cu:93-134) and
    the total rate, energies 1 eV - 20 keV and uniform deviates: FP64 identical to the oracle; FP32 (float
    arguments) identical except where u * total lies within float rounding of a cumulative rate -- the
    cases where the oracle's own choice changes when u moves by 2e-6 -- which are counted and printed."""
    e, h = lines_engine
    b, ho, _ = oracle_lines
    rng = np.random.default_rng(11)
    n = 20000
    E = np.exp(rng.uniform(np.log(1.0), np.log(20000.0), n)) * EV
    u = rng.random(n)
    u[:4] = [0.0, 1.0, 0.5, 1e-9]
    inp = np.column_stack([E, u])
    if prec == FP32:
        inp = np.column_stack([f32_energy(E), f32(u)])
    got = e.eval_pick(h[mat], inp, prec)
    want = oracle_eval(b, "cmo_eval_pick", (ho[mat],), inp, 2)
    live = want[:, 1] > 0
    r = rel(got[live, 1], want[live, 1])
    print("%s prec %d total rate max rel %.3g" % (mat, prec, r.max()))
    assert r.max() < (1e-9 if prec == FP64 else 1e-6)
    same = got[:, 0] == want[:, 0]
    if prec == FP64:
        assert same.all()
        return
    lo, hi = inp.copy(), inp.copy()
    lo[:, 1] *= 1 - 2e-6
    hi[:, 1] = np.minimum(hi[:, 1] * (1 + 2e-6), 1.0)
    edge = oracle_eval(b, "cmo_eval_pick", (ho[mat],), lo, 2)[:, 0] != oracle_eval(b, "cmo_eval_pick", (ho[mat],),
                                                                                   hi, 2)[:, 0]
    for i in np.where(~same)[0][:10]:
        print("  pick differs at E %.9g eV u %.9g: engine %d oracle %d (within rounding: %s)" % (
            inp[i, 0] * FROMSI, inp[i, 1], got[i, 0], want[i, 0], bool(edge[i])))
    print("%s picks within float rounding of a boundary: %d of %d; differing: %d" % (mat, edge.sum(), n,
                                                                                      (~same).sum()))
    assert same[~edge].all()


@pytest.fixture(scope="module")
def phonon_si():
    """Si with GanachaudMokraniPhononInelasticSM (LinesOnLayers.cu:198,205) in an engine and in the oracle."""
    import pyoracle
    from cudamonsel_b200 import capi, scenes
    sc = scenes.halfspace(phonon=True)
    e = capi.Engine(0)
    h = scenes.build_engine(sc, e)
    b, ho = pyoracle.build_oracle(sc)
    yield e, h, b, ho
    e.close()


@pytest.mark.parametrize("prec", [FP64, FP32], ids=["fp64", "fp32"])
def test_phonon(phonon_si, prec):
    """GanachaudMokraniPhononInelasticSM rate and scatter (JMONSEL/GanachaudMokraniPhononInelasticSM.cu:19-72):
    rate, energy after the event, the step's starting energy, the deflected direction and the number of
    deviates drawn (0 below the phonon energy, 2 otherwise).  FP64 against the reference's golden vectors:
    values within 1e-9 relative, directions within 1e-9.  FP32 against the oracle on float-rounded
    inputs: values within 1e-6 relative, directions within 1e-6."""
    e, h, b, ho = phonon_si
    rows = golden("phonon")
    inp = np.ascontiguousarray(rows[:, 0:5])
    if prec == FP64:
        ref = rows[:, 5:11]
        tol_v, tol_d = 1e-9, 1e-9
    else:
        inp = np.column_stack([f32_energy(inp[:, 0]), f32(inp[:, 1:5])])
        ref = oracle_eval(b, "cmo_eval_phonon", (ho["si"], 2), inp, 6)
        tol_v, tol_d = 1e-6, 1e-6
    out = e.eval_phonon(h["si"], 2, inp, prec)
    # the rate (1/m) is 0 below the phonon energy on both sides
    assert ((out[:, 0] == 0) == (ref[:, 0] == 0)).all()
    nz = ref[:, 0] > 0
    for k, j, name in ((0, 0, "rate"), (1, 1, "E"), (5, 4, "Eprev")):
        r = rel(out[nz, k], ref[nz, j]) if name == "rate" else rel(out[:, k], ref[:, j])
        print("phonon %s prec %d max rel %.3g" % (name, prec, r.max()))
        assert r.max() < tol_v, name
    d_ref = unit(ref[:, 2], ref[:, 3])
    dd = np.abs(out[:, 2:5] - d_ref).max(axis=1)
    print("phonon direction prec %d max abs %.3g" % (prec, dd.max()))
    assert dd.max() < tol_d
    # events below the phonon energy change nothing; the others lose exactly one phonon energy
    below = ref[:, 5] == 0
    assert below.any() and (~below).any()
    assert rel(out[below, 1], inp[below, 0]).max() < tol_v


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_csd_fitted_polaron(lines_engine, oracle_lines, prec):
    """JoyLuoNieminenCSD::compute and the FittedInelSM / polaron rates of PMMA."""
    e, h = lines_engine
    b, ho, _ = oracle_lines
    rows = np.array([[float(x) for x in l] for l in golden_lines("pmma", "csd")])
    inp = np.ascontiguousarray(rows[:, 0:2])
    if prec == FP64:
        ref = rows[:, 2:5]
    else:
        inp = np.column_stack([f32_energy(inp[:, 0]), f32(inp[:, 1] * 1e9) / 1e9])
        ref = oracle_eval(b, "cmo_eval_pmma", (ho["pmma"],), inp, 3)
    out = e.eval_csd(h["pmma"], inp, prec)
    for k, name in enumerate(("csd", "fitted", "polaron")):
        r = rel(out[:, k], ref[:, k])
        print("%s prec %d max rel %.3g, 99.9%% %.3g" % (name, prec, r.max(), np.quantile(r, 0.999)))
        assert r.max() < (1e-9 if prec == FP64 else 1e-6)


def test_shapes(engine):
    """NormalMultiPlaneShape / NormalIntersectionShape first normal and containment (double)."""
    from cudamonsel_b200 import scenes
    s = scenes.SceneSpec()
    half = s.planes([0, 0, -1.0], [0, 0, 0])
    c, hh = (5e-9, -3e-9, 12e-9), (15e-9, 10e-9, 5e-9)
    n, p = [], []
    for a in range(3):
        for sg in (-1, 1):
            nn = [0.0, 0.0, 0.0]
            pp = list(c)
            nn[a] = float(sg)
            pp[a] += sg * hh[a]
            n += nn
            p += pp
    block = s.planes(n, p)
    th = 3 * 3.14159265358979323846 / 180
    line = s.line(-100e-9, 40e-9, 1e-6, th, th)
    s.translate(line, [25e-9, 0, 0])
    line0 = s.line(-100e-9, 40e-9, 1e-6, th, th)
    res = scenes.replay(s, scenes.EngineBackend(engine))
    handles = [res[half.idx], res[block.idx], res[line.idx], res[line0.idx]]
    g = golden("shapes")
    for k, sh in enumerate(handles):
        rows = g[g[:, 0] == k]
        out = engine.eval_shape(sh, np.ascontiguousarray(rows[:, 1:7]))
        fin = np.isfinite(rows[:, 10])
        assert (np.isfinite(out[:, 3]) == fin).all()
        assert (out[fin, 0:3] == rows[fin, 7:10]).all()
        r = rel(out[fin, 3], rows[fin, 10])
        print("shape %d u max rel %.3g" % (k, r.max() if fin.any() else 0))
        assert r.max() < 1e-12
        inside = (out[:, 4] == rows[:, 11]).mean()
        print("shape %d containment agreement %.6f" % (k, inside))
        assert inside == 1.0


@pytest.mark.parametrize("fixes", [0, 1])
def test_shapes2(fixes):
    """NormalCylindricalShape, NormalUnionShape and the rounded createLine against the reference's
    own results (cases 0-4: cylinders as the reference builds them; 5-7: axis normalised, built
    here with CM_OPT_JMONSEL_FIXES).  The engine works in nm, the reference in m: u within 1e-9
    relative and normals within 1e-9 where both report a crossing, crossing/containment decisions
    identical."""
    from conftest import shapes2_scene
    from cudamonsel_b200 import capi, scenes
    s, shapes = shapes2_scene(fixes)
    e = capi.Engine(0)
    res = scenes.replay(s, scenes.EngineBackend(e))
    g = golden("shapes2")
    cases = range(5) if fixes == 0 else range(5, 8)
    for k in cases:
        sh = res[shapes[k if fixes == 0 else k - 5].idx]
        rows = g[g[:, 0] == k]
        out = e.eval_shape(sh, np.ascontiguousarray(rows[:, 1:7]))
        fin = np.isfinite(rows[:, 10])
        both = fin & np.isfinite(out[:, 3])
        agree = (np.isfinite(out[:, 3]) == fin).mean()
        r = rel(out[both, 3], rows[both, 10])
        nerr = np.abs(out[both, 0:3] - rows[both, 7:10]).max(axis=1) if both.any() else np.zeros(1)
        print("case %d crossings %d agree %.5f u max rel %.3g normal max err %.3g" % (
            k, fin.sum(), agree, r.max() if both.any() else 0, nerr.max()))
        inside = ((out[:, 4] == rows[:, 11]).mean(), (out[:, 5] == rows[:, 12]).mean())
        print("case %d containment agreement %.6f %.6f" % (k, inside[0], inside[1]))
        assert agree == 1.0
        if both.any():
            assert r.max() < 1e-9 and nerr.max() < 1e-9
        assert inside == (1.0, 1.0)
    e.close()


def test_rotate_shapes():
    """ITransform::rotate (cm_shape_rotate) against the reference's own rotated shapes: blocks rotated with
    both forms of the Euler matrix, a tilted half-space, a cylinder rotated once (which normalises the
    reference's cylinder axis) and twice.  The engine works in nm, the reference in m: u within 1e-9
    relative and normals within 1e-9 where both report a crossing, crossing/containment decisions identical."""
    from conftest import rotate_scene
    from cudamonsel_b200 import capi, scenes
    s, shapes = rotate_scene()
    e = capi.Engine(0)
    res = scenes.replay(s, scenes.EngineBackend(e))
    g = golden("rotate")
    for k, shp in enumerate(shapes):
        rows = g[g[:, 0] == k]
        out = e.eval_shape(res[shp.idx], np.ascontiguousarray(rows[:, 1:7]))
        fin = np.isfinite(rows[:, 10])
        both = fin & np.isfinite(out[:, 3])
        agree = (np.isfinite(out[:, 3]) == fin).mean()
        r = rel(out[both, 3], rows[both, 10])
        nerr = np.abs(out[both, 0:3] - rows[both, 7:10]).max(axis=1)
        print("rotated shape %d crossings %d agree %.5f u max rel %.3g normal max err %.3g" % (
            k, fin.sum(), agree, r.max(), nerr.max()))
        inside = ((out[:, 4] == rows[:, 11]).mean(), (out[:, 5] == rows[:, 12]).mean())
        print("rotated shape %d containment agreement %.6f %.6f" % (k, inside[0], inside[1]))
        assert fin.sum() > 40 and agree == 1.0
        assert r.max() < 1e-9 and nerr.max() < 1e-9
        assert inside == (1.0, 1.0)
    e.close()


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_barrier(engine, prec):
    """ExpQMBarrierSM (classical) both ways across the vacuum/Si surface."""
    from cudamonsel_b200 import scenes
    sc = scenes.halfspace()
    h = scenes.build_engine(sc, engine)
    rows = golden("barrier")
    for d in (0, 1):
        r = rows[rows[:, 0] == d]
        frm, to = (h["si_region"], h["chamber"]) if d == 0 else (h["chamber"], h["si_region"])
        inp = np.ascontiguousarray(r[:, 1:7])
        if prec == FP32:
            # float-rounded energy and angles; the expected energy shifts by the input rounding only
            inp = np.column_stack([f32_energy(inp[:, 0]), f32(inp[:, 1:3]), inp[:, 3:6]])
            r = r.copy()
            r[:, 7] = np.where(r[:, 7] == r[:, 1], inp[:, 0], r[:, 7] + (inp[:, 0] - r[:, 1]))
        out = engine.eval_barrier(frm, to, inp, prec)
        reg = np.where(out[:, 7] == h["si_region"], 1, 0)
        agree = reg == r[:, 13]
        print("dir %d prec %d region agreement %.5f" % (d, prec, agree.mean()))
        assert agree.all()
        er = np.abs(out[agree, 0] - r[agree, 7]) / np.maximum(np.abs(r[agree, 7]), 0.1 * EV)
        print("energy max rel %.3g" % er.max())
        assert er.max() < (1e-12 if prec == FP64 else 2e-6)
        derr = np.abs(out[agree, 1:4] - unit(r[agree, 8], r[agree, 9])).max()
        print("direction max abs err %.3g" % derr)
        assert derr < (1e-12 if prec == FP64 else 1e-6 + 1e-6)
        perr = np.abs(out[agree, 4:7] - r[agree, 10:13]).max()
        assert perr < 1e-20 if prec == FP64 else perr < 1e-17


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_freepath(engine, prec):
    """MONSEL_MaterialScatterModel::randomMeanPathLength for Si."""
    from cudamonsel_b200 import scenes
    sc = scenes.halfspace()
    h = scenes.build_engine(sc, engine)
    fp = np.array([[float(x) for x in l] for l in golden_lines("misc", "fpath")])
    inp = np.ascontiguousarray(fp[:, 0:2])
    ref = fp[:, 2]
    if prec == FP32:
        import pyoracle
        b, ho = pyoracle.build_oracle(sc)
        inp = np.column_stack([f32_energy(inp[:, 0]), f32(inp[:, 1])])
        ref = oracle_eval(b, "cmo_eval_freepath", (ho["si"],), inp, 1)[:, 0]
    out = engine.eval_freepath(h["si"], inp, prec)
    r = rel(out, ref)
    print("free path prec %d max rel %.3g" % (prec, r.max()))
    assert r.max() < (1e-9 if prec == FP64 else 1e-6)


def test_random_inputs_against_oracle(lines_engine, oracle_lines):
    """Fresh random inputs (not the golden set): FP64 kernels vs the C oracle for the
    inelastic and elastic events across 2 eV - 15 keV."""
    import ctypes as C
    import pyoracle as po
    e, h = lines_engine
    b, ho, _ = oracle_lines
    rng = np.random.default_rng(7)
    n = 20000
    E = np.exp(rng.uniform(np.log(2.0), np.log(15000.0), n)) * EV
    inp = np.column_stack([E, rng.uniform(0, np.pi, n), rng.uniform(-np.pi, np.pi, n), rng.random((n, 6))])
    out = e.eval_tabulated(h["si"], 1, inp, FP64)
    ref = np.zeros((n, 9))
    b.L.cmo_eval_tabulated(b.h, ho["si"], 1, n, po.dp(inp), ref.ctypes.data_as(C.POINTER(C.c_double)))
    assert (out[:, 5] == ref[:, 4]).all()
    assert rel(out[:, 1], ref[:, 1]).max() < 1e-9
    inp2 = np.column_stack([E, rng.uniform(0, np.pi, n), rng.uniform(-np.pi, np.pi, n), rng.random((n, 4))])
    out2 = e.eval_elastic(h["pmma"], 0, inp2, FP64)
    ref2 = np.zeros((n, 5))
    b.L.cmo_eval_elastic(b.h, ho["pmma"], 0, n, po.dp(inp2), ref2.ctypes.data_as(C.POINTER(C.c_double)))
    assert (out2[:, 4] == ref2[:, 3]).all()
    assert np.abs(out2[:, 1:4] - unit(ref2[:, 1], ref2[:, 2])).max() < 1e-8
