"""A stream of scan jobs served by cm_server: seeded random scenes, Poisson arrivals, p50/p99 latency.

The workload follows the served-stream configuration: each job is a Si substrate carrying 1-8 PMMA or
Si features (trapezoid lines from NShapes::createLine or cylinders lying along y) with dimensions
~U(10, 200) nm, a beam energy ~U(200, 5000) eV, and either an image or a linescan, at 100-1000
primaries per pixel.  `scale` shrinks the scan sizes and primary counts together (the full stream is
hours of transport); the distributions keep their shape.
"""
import math
import time

import numpy as np

from . import capi, scenes

IMAGE_SIDES = (32, 64, 128, 256)


def job_scene(rng, spec=None):
    """One job's geometry: 1-8 features on Si, materials as LinesOnLayers.cu.  Cylinders are built with
    their axis normalised (the reference's as-compiled cylinders are never struck)."""
    s = spec or scenes.SceneSpec()
    vac = scenes.vacuum(s)
    si = scenes.silicon(s)
    pm = scenes.pmma(s)
    chamber = s.region(None, vac, s.sphere([0.0, 0.0, 0.0], 0.1))
    surf = s.planes([0.0, 0.0, -1.0], [0.0, 0.0, 0.0])
    s.region(chamber, si, surf)
    nfeat = int(rng.integers(1, 9))
    x = -0.5e-6
    top = 0.0
    for _ in range(nfeat):
        size = rng.uniform(10e-9, 200e-9)
        height = rng.uniform(10e-9, 200e-9)
        msm = pm if rng.random() < 0.5 else si
        if rng.random() < 0.5:
            th = math.radians(rng.uniform(0.0, 10.0))
            shp = s.line(-height, size, 2e-6, th, th)
            s.translate(shp, [x + size / 2, 0.0, 0.0])
            top = max(top, height)
        else:
            r = size / 2
            s.set_options(1)
            shp = s.cylinder([x + r, -1e-6, -r], [x + r, 1e-6, -r], r)
            s.set_options(0)
            top = max(top, size)
        s.region(chamber, msm, shp)
        x += size + rng.uniform(10e-9, 100e-9)
    return s, chamber, top


def job_scan(rng, scale=1.0, top=100e-9):
    """Pixel centres (the beam starts 20 nm above the tallest feature), beam energy (J), primaries per
    pixel and bins of one job."""
    z0 = -max(120e-9, top + 20e-9)
    energy_eV = rng.uniform(200.0, 5000.0)
    nprim = max(1, int(rng.integers(100, 1001) * scale))
    if rng.random() < 0.5:
        side = max(2, int(IMAGE_SIDES[int(rng.integers(0, 4))] * math.sqrt(scale)))
        step = 2e-9
        xs = (np.arange(side) - (side - 1) / 2.0) * step
        gx, gy = np.meshgrid(xs, xs)
        centers = np.stack([gx.ravel(), gy.ravel(), np.full(side * side, z0)], axis=1)
    else:
        npix = max(2, int(rng.integers(64, 513) * scale))
        xs = (np.arange(npix) - (npix - 1) / 2.0) * 1e-9
        centers = np.stack([xs, np.zeros(npix), np.full(npix, z0)], axis=1)
    nbins = max(1, int(energy_eV / 10.0))
    return centers, scenes.eV(energy_eV), nprim, nbins


def make_jobs(n, seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n):
        spec, chamber, top = job_scene(rng)
        centers, energy, nprim, nbins = job_scan(rng, scale, top)
        keys = np.arange(len(centers), dtype=np.uint64) + np.uint64((k + 1) * 1_000_003)
        jobs.append(dict(spec=spec, chamber=chamber, centers=centers, energy=energy, nprim=nprim, nbins=nbins,
                         keys=keys))
    return jobs


def submit(server, holder, job, precision=capi.PREC_FP32):
    """Describe the job's scene in `holder` (an Engine used only as a scene registry) and queue it."""
    holder.reset()
    res = scenes.replay(job["spec"], scenes.EngineBackend(holder))
    return server.submit(holder, res[job["chamber"].idx], job["centers"], job["energy"], job["nprim"], job["nbins"],
                         1e-9, 0, precision, pixel_keys=job["keys"])


def serve(jobs, rate_per_s, slots=4, budget_gb=16.0, seed=1, precision=capi.PREC_FP32, device=0):
    """Submit `jobs` at Poisson arrival times (mean rate_per_s; None: all at once, which saturates the
    server) to a fresh server, wait for all of them; returns per-job latencies (end - submit, s), makespan
    (first submission to last end, s), primaries and electron-steps."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, len(jobs)) if rate_per_s else np.zeros(len(jobs))
    server = capi.Server(device, slots, budget_gb)
    holder = capi.Engine(device)
    ids = []
    t0 = time.perf_counter()
    due = 0.0
    for job, gap in zip(jobs, gaps):
        due += gap
        wait = due - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        ids.append(submit(server, holder, job, precision))
    infos = [server.wait(j) for j in ids]
    bad = [(j, i.state) for j, i in zip(ids, infos) if i.state != capi.JOB_DONE]
    results = [server.result(j) for j in ids] if not bad else []
    why = ""
    if bad:
        try:
            server.result(bad[0][0])
        except capi.CMError as e:
            why = str(e)
    server.close()
    holder.close()
    if bad:
        raise capi.CMError("%d jobs did not complete (states %s): %s" % (len(bad), sorted({s for _, s in bad}), why))
    lat = np.array([i.end_s - i.submit_s for i in infos])
    first = min(i.submit_s for i in infos)
    makespan = max(i.end_s for i in infos) - first
    prim = sum(int(i.primaries) for i in infos)
    steps = sum(int(i.steps) for i in infos)
    return dict(latency=lat, makespan=makespan, primaries=prim, steps=steps, results=results, infos=infos)
