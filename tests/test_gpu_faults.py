"""Failures made on the host or by the caller's inputs, on the GPU: each returns a status, nothing faults,
and the context keeps working.  A table with a non-finite or non-monotonic axis, or a non-finite value, is
refused by cm_add_table; a pixel with a NaN or infinite energy or a non-finite centre by cm_run; a job
cancelled while its loop runs on the device ends CANCELLED at its next iteration and the slot serves the
next job; the counters of electrons ended by the zero-energy cut and the step limit are reported."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def half():
    from cudamonsel_b200 import capi, scenes
    e = capi.Engine(0)
    h = scenes.build_engine(scenes.halfspace(), e)
    yield e, h
    e.close()


def normal_run(e, h):
    from cudamonsel_b200 import scenes
    b, f, st = e.run(h["chamber"], np.array([[0.0, 0.0, -20e-9]]), scenes.eV(1000.0), 200, 100, 0.0, 5)
    assert st.primaries == 200 and b.sum() > 0
    return st


def test_corrupt_tables_are_refused(half):
    from cudamonsel_b200 import capi
    e, h = half
    x = np.array([1.0, 2.0, 3.0, 4.0, 5.0])
    v = np.arange(5.0)
    for axis, vals, what in ((np.array([1.0, 2.0, np.nan, 4.0, 5.0]), v, "non-finite"),
                             (np.array([1.0, 3.0, 2.0, 4.0, 5.0]), v, "monotonic"),
                             (x, np.array([0.0, 1.0, np.inf, 3.0, 4.0]), "value not finite")):
        with pytest.raises(capi.CMError, match=what) as ei:
            e.table(1, [5], [axis], vals)
        assert ei.value.code == capi.EINVAL
    normal_run(e, h)


def test_bad_pixels_are_refused(half):
    from cudamonsel_b200 import capi, scenes
    e, h = half
    c = np.array([[0.0, 0.0, -20e-9]])
    for energy, centre in ((np.nan, c), (np.inf, c), (-scenes.eV(100.0), c),
                           (scenes.eV(1000.0), np.array([[np.nan, 0.0, -20e-9]])),
                           (scenes.eV(1000.0), np.array([[0.0, np.inf, -20e-9]]))):
        with pytest.raises(capi.CMError) as ei:
            e.run(h["chamber"], centre, energy, 10, 100, 0.0, 1)
        assert ei.value.code == capi.EINVAL
    st = normal_run(e, h)
    assert st.ended_step_limit == 0


def test_cancel_a_running_job():
    """A job of 2M primaries at 2 keV takes seconds; cancelled once it runs, the device loop sees the flag at
    its next iteration: the job ends CANCELLED well before it could have finished, and the slot then runs
    the next job to the end."""
    import time
    from cudamonsel_b200 import capi, scenes
    srv = capi.Server(0, slots=1, budget_gb=8.0)
    holder = capi.Engine(0)
    h = scenes.build_engine(scenes.halfspace(), holder)
    centers = np.tile([0.0, 0.0, -20e-9], (200, 1))
    big = srv.submit(holder, h["chamber"], centers, scenes.eV(2000.0), 10000, 200, 0.0, 3)
    t0 = time.time()
    while srv.poll(big).state == capi.JOB_QUEUED and time.time() - t0 < 60:
        time.sleep(0.005)
    time.sleep(0.05)
    srv.cancel(big)
    info = srv.wait(big, 60.0)
    print("cancelled job: state %d after %.3f s of running" % (info.state, info.end_s - info.start_s))
    assert info.state == capi.JOB_CANCELLED and info.error == capi.ECANCELED
    small = srv.submit(holder, h["chamber"], centers[:4], scenes.eV(1000.0), 100, 100, 0.0, 4)
    assert srv.wait(small, 60.0).state == capi.JOB_DONE
    srv.close()
    holder.close()


def test_ended_electron_counters_are_reported(half):
    """The counts of electrons ended by the zero-energy cut (no energy left in a region without mechanisms,
    ended after 4096 steps) and by the step limit come back with the run's statistics (flat Si at 1 keV
    ends none either way)."""
    e, h = half
    st = normal_run(e, h)
    d = st.as_dict()
    print("ended by the zero-energy cut: %d, by the step limit: %d" % (d["ended_zero_energy"], d["ended_step_limit"]))
    assert d["ended_zero_energy"] == 0 and d["ended_step_limit"] == 0
