"""Host logic of scan.run_checkpointed (no GPU): parts, the checkpoint file, resuming, and refusing another
scan's checkpoint, driven by a stand-in engine whose tallies, like the engine's, depend only on each
pixel's key and primary indices and add up over primaries."""
import numpy as np
import pytest


class CountingEngine:
    """Engine.run's signature; primary k of pixel p lands in bin (key_p * 31 + k * 7) mod (nbins + 2) of the
    back histogram and in the fwd histogram's bin 0 when k is odd."""

    def __init__(self):
        self.calls = []

    def run(self, chamber, centers, energies, nprim, nbins, beam_width, seed, precision=0, pixel_keys=None,
            first_primary=None):
        npix = len(centers)
        stride = int(np.max(nbins)) + 2
        back = np.zeros((npix, stride), dtype=np.uint32)
        fwd = np.zeros((npix, stride), dtype=np.uint32)
        first = np.zeros(npix, dtype=np.int64) if first_primary is None else np.asarray(first_primary)
        for p in range(npix):
            for k in range(int(first[p]), int(first[p]) + int(nprim[p])):
                back[p, (int(pixel_keys[p]) * 31 + k * 7) % stride] += 1
                fwd[p, 0] += k & 1
        self.calls.append((np.asarray(nprim).copy(), first.copy()))
        return back, fwd, None


def inputs():
    centers = np.zeros((5, 3))
    nprim = np.array([700, 0, 1, 250, 501], dtype=np.int32)
    keys = np.arange(5, dtype=np.uint64) + np.uint64(3)
    return centers, nprim, keys


def test_parts_equal_one_call_and_resume(tmp_path):
    from cudamonsel_b200 import scan
    centers, nprim, keys = inputs()
    e = CountingEngine()
    back, fwd, _ = e.run(0, centers, 1.0, nprim, 20, 0.0, 0, pixel_keys=keys)
    e = CountingEngine()
    b, f, done = scan.run_checkpointed(e, 0, centers, 1.0, nprim, 20, 0.0, 0, keys, part=250)
    assert np.array_equal(done, nprim) and len(e.calls) == 3
    assert np.array_equal(b, back.astype(np.uint64)) and np.array_equal(f, fwd.astype(np.uint64))
    # each part starts where the last ended and takes at most `part` primaries per pixel
    assert np.array_equal(e.calls[1][1], np.minimum(nprim, 250))
    assert (np.stack([c[0] for c in e.calls]) <= 250).all()
    ck = str(tmp_path / "scan.npz")
    e = CountingEngine()
    _, _, d1 = scan.run_checkpointed(e, 0, centers, 1.0, nprim, 20, 0.0, 0, keys, part=250, checkpoint=ck, max_parts=2)
    assert np.array_equal(d1, np.minimum(nprim, 500)) and len(e.calls) == 2
    e = CountingEngine()
    b2, f2, d2 = scan.run_checkpointed(e, 0, centers, 1.0, nprim, 20, 0.0, 0, keys, part=250, checkpoint=ck)
    assert len(e.calls) == 1 and np.array_equal(d2, nprim)  # only the last part is run
    assert np.array_equal(b2, back.astype(np.uint64)) and np.array_equal(f2, fwd.astype(np.uint64))
    e = CountingEngine()
    scan.run_checkpointed(e, 0, centers, 1.0, nprim, 20, 0.0, 0, keys, part=250, checkpoint=ck)
    assert not e.calls  # a finished checkpoint runs nothing more


def test_another_scans_checkpoint_is_refused(tmp_path):
    from cudamonsel_b200 import scan
    centers, nprim, keys = inputs()
    ck = str(tmp_path / "scan.npz")
    scan.run_checkpointed(CountingEngine(), 0, centers, 1.0, nprim, 20, 0.0, 0, keys, part=250, checkpoint=ck,
                          max_parts=1)
    with pytest.raises(ValueError):
        scan.run_checkpointed(CountingEngine(), 0, centers, 1.0, nprim + 1, 20, 0.0, 0, keys, checkpoint=ck)
    with pytest.raises(ValueError):
        scan.run_checkpointed(CountingEngine(), 0, centers, 1.0, nprim, 20, 0.0, 0, keys + np.uint64(1),
                              checkpoint=ck)
