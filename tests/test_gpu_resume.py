"""Checkpoint/resume of a scan: a scan run in parts (cm_run_desc.pixel_first = primaries already done) gives
the tallies of one run over the whole scan, count for count, in both precisions; a scan interrupted after
its first part carries on from its checkpoint file; the entry points that do not take pixel_first refuse it."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lines():
    from cudamonsel_b200 import capi, scenes
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.lines(), e)
    yield e, h
    e.close()


def scan_inputs():
    from cudamonsel_b200 import scenes
    centers = scenes.linescan_pixels(16, 8e-9, 0.0, -120e-9)
    nprim = np.array([600, 0, 1, 250, 251, 599] + [500] * 10, dtype=np.int32)  # ragged, an empty pixel
    keys = np.arange(16, dtype=np.uint64) * np.uint64(7919) + np.uint64(31)
    return centers, nprim, keys


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32"])
def test_parts_add_up_to_one_run(lines, prec, tmp_path):
    from cudamonsel_b200 import scan, scenes
    e, h = lines
    centers, nprim, keys = scan_inputs()
    back, fwd, st = e.run(h["chamber"], centers, scenes.eV(500.0), nprim, 50, 1e-9, 0, precision=prec,
                          pixel_keys=keys)
    pb, pf, done = scan.run_checkpointed(e, h["chamber"], centers, scenes.eV(500.0), nprim, 50, 1e-9, prec, keys,
                                         part=250)
    assert np.array_equal(done, nprim)
    assert np.array_equal(pb, back.astype(np.uint64)) and np.array_equal(pf, fwd.astype(np.uint64))
    print("prec %d: %d primaries in 3 parts, %d back counts: identical to one run" % (prec, nprim.sum(), back.sum()))
    # interrupted after its first part, then resumed from the checkpoint file
    ck = str(tmp_path / "scan.npz")
    b1, _, d1 = scan.run_checkpointed(e, h["chamber"], centers, scenes.eV(500.0), nprim, 50, 1e-9, prec, keys,
                                      part=250, checkpoint=ck, max_parts=1)
    assert (d1 == np.minimum(nprim, 250)).all() and b1.sum() < back.sum()
    rb, rf, rd = scan.run_checkpointed(e, h["chamber"], centers, scenes.eV(500.0), nprim, 50, 1e-9, prec, keys,
                                       part=250, checkpoint=ck)
    assert np.array_equal(rd, nprim)
    assert np.array_equal(rb, back.astype(np.uint64)) and np.array_equal(rf, fwd.astype(np.uint64))
    with pytest.raises(ValueError):  # a checkpoint of another scan is not taken
        scan.run_checkpointed(e, h["chamber"], centers, scenes.eV(500.0), nprim, 50, 1e-9, prec, keys + np.uint64(1),
                              part=250, checkpoint=ck)


def test_pixel_first_refused_where_not_taken(lines):
    import torch
    from cudamonsel_b200 import capi, scenes
    e, h = lines
    centers, nprim, keys = scan_inputs()
    e.run(h["chamber"], centers, scenes.eV(500.0), 1, 50, 1e-9, 0, precision=capi.PREC_FP32, pixel_keys=keys)
    dev = torch.device("cuda", 0)
    t_c = torch.tensor(centers.ravel(), dtype=torch.float64, device=dev)
    t_e = torch.full((16,), scenes.eV(500.0), dtype=torch.float64, device=dev)
    t_n = torch.tensor(nprim, dtype=torch.int32, device=dev)
    t_b = torch.full((16,), 50, dtype=torch.int32, device=dev)
    t_first = torch.zeros(16, dtype=torch.int64, device=dev)
    back = torch.zeros((16, 52), dtype=torch.int32, device=dev)
    fwd = torch.zeros_like(back)
    P = lambda t, ty: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ty))
    d = capi.RunDesc(h["chamber"], capi.PREC_FP32, 16, 1e-9, P(t_c, C.c_double), P(t_e, C.c_double), P(t_n, C.c_int),
                     P(t_b, C.c_int), 0, 52, 0, 0, None, 0)
    d.pixel_first = P(t_first, C.c_int64)
    with pytest.raises(capi.CMError) as err:
        e.run_noalloc(d, back.data_ptr(), fwd.data_ptr())
    assert err.value.code == capi.EINVAL and "pixel_first" in str(err.value)
    # cm_run_device takes it (device array): all zero is the same as none
    st = e.run_device(d, back.data_ptr(), fwd.data_ptr())
    torch.cuda.synchronize()
    b0, _, _ = e.run(h["chamber"], centers, scenes.eV(500.0), nprim, 50, 1e-9, 0, precision=capi.PREC_FP32)
    assert st.primaries == int(nprim.sum())
    assert np.array_equal(back.cpu().numpy().astype(np.uint32), b0)
