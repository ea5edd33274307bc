"""cm_run_noalloc, the allocation-free transport run, against cm_run_device.

Every electron's random stream is keyed by its lineage, so the tallies do not
depend on the wave size or batch: the allocation-free run (smaller wave, fixed
scratch) must give exactly the histograms cm_run_device gives for the same
inputs -- the tolerance is zero, as in the determinism tests.  Two calls in a
row, with different inputs, check that the second does not see what the first
left in the shared scratch.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64, FP32 = 0, 1


@pytest.fixture(scope="module")
def setup():
    import torch
    from cudamonsel_b200 import capi, scenes
    e = capi.Engine(0)
    sc = scenes.lines()
    h = scenes.build_engine(sc, e)
    yield torch, capi, scenes, e, h
    e.close()


def inputs(torch, scenes, npix, nprim, beam_eV, key0):
    dev = torch.device("cuda", 0)
    x = np.linspace(-150e-9, 150e-9, npix)
    centers = np.stack([x, np.zeros(npix), np.full(npix, -120e-9)], axis=1)
    nb = int(beam_eV / 10)
    return dict(
        center=torch.tensor(centers.ravel(), dtype=torch.float64, device=dev),
        energy=torch.full((npix,), scenes.eV(beam_eV), dtype=torch.float64, device=dev),
        nprim=torch.tensor([nprim + (i % 3) for i in range(npix)], dtype=torch.int32, device=dev),
        nbins=torch.full((npix,), nb, dtype=torch.int32, device=dev),
        keys=torch.arange(key0, key0 + npix, dtype=torch.int64, device=dev),
        npix=npix, stride=nb + 2)


def desc(capi, h, t, prec):
    P = lambda x, ty: C.cast(C.c_void_p(x.data_ptr()), C.POINTER(ty))
    return capi.RunDesc(h["chamber"], prec, t["npix"], 1e-9, P(t["center"], C.c_double), P(t["energy"], C.c_double),
                        P(t["nprim"], C.c_int), P(t["nbins"], C.c_int), 0, t["stride"], 0, 0,
                        P(t["keys"], C.c_uint64), 0)


def tallies(torch, t):
    z = lambda: torch.full((t["npix"], t["stride"]), 7, dtype=torch.int32, device=t["center"].device)
    return z(), z()  # non-zero on purpose: the run must clear them


@pytest.mark.parametrize("prec", [FP32, FP64])
def test_noalloc_matches_run_device_twice(setup, prec):
    torch, capi, scenes, e, h = setup
    cases = [inputs(torch, scenes, 48, 60, 500.0, 1000), inputs(torch, scenes, 17, 90, 800.0, 5000)]
    want = []
    for t in cases:
        b, f = tallies(torch, t)
        st = e.run_device(desc(capi, h, t, prec), b.data_ptr(), f.data_ptr())
        torch.cuda.synchronize()
        want.append((b.cpu().numpy(), f.cpu().numpy(), st.steps, st.primaries))
    got = []
    for t in cases:  # two allocation-free calls in a row
        b, f = tallies(torch, t)
        st = e.run_noalloc(desc(capi, h, t, prec), b.data_ptr(), f.data_ptr())
        torch.cuda.synchronize()
        got.append((b.cpu().numpy(), f.cpu().numpy(), st.steps, st.primaries))
    for (wb, wf, ws, wp), (gb, gf, gs, gp), t in zip(want, got, cases):
        assert gp == wp == int(t["nprim"].sum())
        assert wb.sum() > 0
        np.testing.assert_array_equal(gb, wb)
        np.testing.assert_array_equal(gf, wf)
        assert gs == ws


def test_noalloc_rejects_too_many_pixels(setup):
    torch, capi, scenes, e, h = setup
    t = inputs(torch, scenes, 65537, 1, 500.0, 1)
    b, f = tallies(torch, t)
    with pytest.raises(capi.CMError, match="exceeds its maximum of 65536"):
        e.run_noalloc(desc(capi, h, t, FP32), b.data_ptr(), f.data_ptr())


def test_noalloc_allocates_nothing(setup):
    """After a first call (which looks up the scratch array's address), further calls leave the device's
    free memory exactly where it was: nothing is allocated, not even transiently kept."""
    torch, capi, scenes, e, h = setup
    t = inputs(torch, scenes, 32, 80, 500.0, 77)
    b, f = tallies(torch, t)
    e.run_noalloc(desc(capi, h, t, FP32), b.data_ptr(), f.data_ptr())
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(2):
        e.run_noalloc(desc(capi, h, t, FP32), b.data_ptr(), f.data_ptr())
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0


def test_noalloc_rejects_bad_input_and_missing_scene(setup):
    """A negative primary count is CM_EINVAL (checked on the device before any transport); a context whose
    scene was never uploaded for the precision is CM_ESTATE (uploading would allocate)."""
    torch, capi, scenes, e, h = setup
    t = inputs(torch, scenes, 8, 10, 500.0, 3)
    t["nprim"][3] = -1
    b, f = tallies(torch, t)
    with pytest.raises(capi.CMError, match="negative primary count") as ei:
        e.run_noalloc(desc(capi, h, t, FP32), b.data_ptr(), f.data_ptr())
    assert ei.value.code == capi.EINVAL
    fresh = capi.Engine(0)
    try:
        hf = scenes.build_engine(scenes.lines(), fresh)
        t = inputs(torch, scenes, 8, 10, 500.0, 3)
        with pytest.raises(capi.CMError) as ei:
            fresh.run_noalloc(desc(capi, hf, t, FP64), b.data_ptr(), f.data_ptr())
        assert ei.value.code == capi.ESTATE
    finally:
        fresh.close()


def test_noalloc_stops_with_a_status_and_the_scratch_recovers(setup):
    """A call that hits its iteration limit (desc.max_iterations = 16, far fewer than the run needs) returns
    CM_ELIMIT with electrons still in the shared scratch; the next call clears what must start at zero and
    gives cm_run_device's tallies again."""
    torch, capi, scenes, e, h = setup
    t = inputs(torch, scenes, 24, 50, 500.0, 4242)
    b, f = tallies(torch, t)
    d = desc(capi, h, t, FP32)
    d.max_iterations = 16
    with pytest.raises(capi.CMError, match="iteration limit") as ei:
        e.run_noalloc(d, b.data_ptr(), f.data_ptr())
    assert ei.value.code == capi.ELIMIT
    b, f = tallies(torch, t)
    e.run_device(desc(capi, h, t, FP32), b.data_ptr(), f.data_ptr())
    torch.cuda.synchronize()
    want = b.cpu().numpy()
    b, f = tallies(torch, t)
    e.run_noalloc(desc(capi, h, t, FP32), b.data_ptr(), f.data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(b.cpu().numpy(), want)
