"""The job server (cm_server): a job's tallies are the same alone, in a mix of concurrent jobs and
through cm_run; queued and running jobs can be cancelled; admission is first in, first out under the
device-memory budget; a Poisson stream of random scan jobs completes with its latencies reported.
Tallies are integer counts keyed by per-pixel random streams, so "the same" means identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def jobs():
    from cudamonsel_b200 import serving
    return serving.make_jobs(6, seed=3, scale=1 / 32)


def test_job_same_alone_in_mix_and_through_cm_run(jobs):
    from cudamonsel_b200 import capi, scenes, serving
    srv = capi.Server(0, slots=3, budget_gb=8.0)
    holder = capi.Engine(0)
    alone = serving.submit(srv, holder, jobs[0])
    info = srv.wait(alone)
    assert info.state == capi.JOB_DONE and info.primaries == len(jobs[0]["centers"]) * jobs[0]["nprim"]
    b0, f0, _ = srv.result(alone)
    ids = [serving.submit(srv, holder, j) for j in jobs]
    infos = [srv.wait(j) for j in ids]
    assert all(i.state == capi.JOB_DONE for i in infos)
    # the jobs overlapped on the device: some job started before another ended
    spans = sorted((i.start_s, i.end_s) for i in infos)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))
    res = [srv.result(j) for j in ids]
    assert (res[0][0] == b0).all() and (res[0][1] == f0).all()
    srv.close()
    # the same job through cm_run on an engine of its own
    j = jobs[0]
    e = capi.Engine(0)
    h = scenes.replay(j["spec"], scenes.EngineBackend(e))
    back, fwd, st = e.run(h[j["chamber"].idx], j["centers"], j["energy"], j["nprim"], j["nbins"], 1e-9, 0,
                          precision=capi.PREC_FP32, pixel_keys=j["keys"])
    e.close()
    holder.close()
    assert (back == b0).all() and (fwd == f0).all()


def test_precisions_batch_apart_and_match_cm_run(jobs):
    """FP32 and FP64 jobs submitted together run in two batches at once; each job's tallies are those of
    cm_run at its precision, and FP32 is the same whether its neighbours in the batch came first or not."""
    from cudamonsel_b200 import capi, scenes, serving
    srv = capi.Server(0, slots=8, budget_gb=8.0)
    holder = capi.Engine(0)
    precs = [capi.PREC_FP32, capi.PREC_FP64, capi.PREC_FP32, capi.PREC_FP64]
    ids = [serving.submit(srv, holder, j, p) for j, p in zip(jobs[2:6], precs)]
    infos = [srv.wait(j) for j in ids]
    assert all(i.state == capi.JOB_DONE for i in infos)
    res = [srv.result(j) for j in ids]
    e = capi.Engine(0)
    for j, p, (b, f, st) in zip(jobs[2:6], precs, res):
        e.reset()
        h = scenes.replay(j["spec"], scenes.EngineBackend(e))
        back, fwd, rs = e.run(h[j["chamber"].idx], j["centers"], j["energy"], j["nprim"], j["nbins"], 1e-9, 0,
                              precision=p, pixel_keys=j["keys"])
        assert (back == b).all() and (fwd == f).all()
        assert st.primaries == rs.primaries and st.steps == rs.steps
    e.close()
    # the second FP32 job alone in a fresh server: the same as in the mix
    j = jobs[4]
    alone = serving.submit(srv, holder, j, capi.PREC_FP32)
    assert srv.wait(alone).state == capi.JOB_DONE
    b, f, _ = srv.result(alone)
    assert (b == res[2][0]).all() and (f == res[2][1]).all()
    srv.close()
    holder.close()


def test_cancel_queued_and_running(jobs):
    from cudamonsel_b200 import capi, serving
    srv = capi.Server(0, slots=1, budget_gb=8.0)
    holder = capi.Engine(0)
    big = dict(jobs[1])
    big["nprim"] = 20000
    running = serving.submit(srv, holder, big)
    queued = serving.submit(srv, holder, jobs[2])
    srv.cancel(queued)
    assert srv.poll(queued).state == capi.JOB_CANCELLED
    while srv.poll(running).state == capi.JOB_QUEUED:
        pass
    srv.cancel(running)
    info = srv.wait(running, 60.0)
    assert info.state in (capi.JOB_CANCELLED, capi.JOB_DONE)
    with pytest.raises(capi.CMError):
        srv.result(queued)
    after = serving.submit(srv, holder, jobs[3])  # the slot serves the next job normally
    assert srv.wait(after).state == capi.JOB_DONE
    srv.close()
    holder.close()


def test_budget_admits_first_in_first_out(jobs):
    from cudamonsel_b200 import capi, serving
    # a budget below any job's footprint: a job starts only when nothing else runs, in submission order
    srv = capi.Server(0, slots=3, budget_gb=1e-9)
    holder = capi.Engine(0)
    ids = [serving.submit(srv, holder, j) for j in jobs[:4]]
    infos = [srv.wait(j) for j in ids]
    for a, b in zip(infos, infos[1:]):
        assert b.start_s >= a.end_s - 1e-6
    srv.close()
    holder.close()


def test_poisson_stream_latencies():
    from cudamonsel_b200 import serving
    js = serving.make_jobs(12, seed=11, scale=1 / 32)
    out = serving.serve(js, rate_per_s=40.0, slots=4, budget_gb=8.0)
    lat = out["latency"]
    assert len(lat) == 12 and (lat > 0).all()
    print("p50 %.3f s p99 %.3f s makespan %.2f s %d primaries" % (np.percentile(lat, 50), np.percentile(lat, 99),
                                                                 out["makespan"], out["primaries"]))


def test_jobs_on_one_sample_share_its_geometry_and_match_cm_run():
    """Jobs with the same geometry (a linescan split into bands with keys of their own, and a job on another
    sample between them) share one chamber in the batch's scene; each job's tallies are those of cm_run on
    its own."""
    from cudamonsel_b200 import capi, scenes
    sc = scenes.lines()
    holder = capi.Engine(0)
    h = scenes.build_engine(sc, holder)
    other = capi.Engine(0)
    ho = scenes.build_engine(scenes.halfspace(), other)
    centers = scenes.linescan_pixels(48, 2e-9, 0.0, -120e-9)
    bands = [slice(0, 16), slice(16, 32), slice(32, 48)]
    keys = np.arange(48, dtype=np.uint64) * np.uint64(104729) + np.uint64(11)
    srv = capi.Server(0, slots=8, budget_gb=8.0)
    ids = [srv.submit(holder, h["chamber"], centers[b], scenes.eV(500.0), 300, 50, 1e-9, 0, capi.PREC_FP32,
                      pixel_keys=keys[b]) for b in bands[:2]]
    ids.append(srv.submit(other, ho["chamber"], centers[:4], scenes.eV(800.0), 300, 80, 1e-9, 0, capi.PREC_FP32,
                          pixel_keys=keys[:4]))
    ids.append(srv.submit(holder, h["chamber"], centers[bands[2]], scenes.eV(500.0), 300, 50, 1e-9, 0,
                          capi.PREC_FP32, pixel_keys=keys[bands[2]]))
    infos = [srv.wait(j) for j in ids]
    assert all(i.state == capi.JOB_DONE for i in infos)
    res = [srv.result(j) for j in ids]
    srv.close()
    back, fwd, _ = holder.run(h["chamber"], centers, scenes.eV(500.0), 300, 50, 1e-9, 0, precision=capi.PREC_FP32,
                              pixel_keys=keys)
    for (b, f, _), band in zip([res[0], res[1], res[3]], bands):
        assert (b == back[band]).all() and (f == fwd[band]).all()
    bo, fo, _ = other.run(ho["chamber"], centers[:4], scenes.eV(800.0), 300, 80, 1e-9, 0, precision=capi.PREC_FP32,
                          pixel_keys=keys[:4])
    assert (res[2][0] == bo).all() and (res[2][1] == fo).all()
    holder.close()
    other.close()
