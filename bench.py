"""Throughput of the electron-transport hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): the linescan -- three PMMA trapezoid lines (height 100 nm,
bottom width 40 nm, 3 deg sidewalls, pitch 200 nm) on a Si substrate, a 500 eV
Gaussian beam (sigma 1 nm) landing on 256 pixels 1 nm apart across the
middle line, 2000 primaries per pixel (512 000 primaries), synthetic tables.
Metric: primary electrons per second, FP32 transport (FP64 positions and
plane solves), with the linescan yields checked against an FP64 run of the
same workload.  Before the warm-up the engine's autotuner picks the launch
settings of each precision on this workload (--no-autotune: defaults); they
are printed in config.tuning.  Under torchrun each rank runs the full linescan
with its own random streams (weak scaling, no collective on the data path);
the time is the max over ranks.  Further lines: the rough-line image (both
precisions autotuned on its first eighth of rows; FP32 batched against the plain
FP64 form at default settings and against FP64 tuned; the image also served as
16 jobs), the 10 keV deep layout (--deep-side 512 --deep-primaries 500 for its
full size) and the served stream (Poisson arrivals and saturated, FP32 and FP64).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NPIX, NPRIM, BEAM_EV, NBINS = 256, 2000, 500.0, 50
METRIC = "primary electrons/s at <=1% BSE/SE yield error vs FP64"
WORKLOAD = ("linescan: 3 PMMA lines (h 100 nm, bottom w 40 nm, 3 deg, pitch 200 nm) on Si, 500 eV Gaussian "
            "sigma 1 nm, 256 px x 1 nm, 2000 primaries/px (512k primaries)")
# served stream (latency line): jobs, mean arrival rate (1/s), server slots and budget, size scale
SERVE_JOBS, SERVE_RATE, SERVE_SLOTS, SERVE_BUDGET_GB, SERVE_SCALE = 64, 8.0, 16, 16.0, 1 / 8
IMAGE_REPEATS = 3  # runs per precision of the rough-line image
IMAGE_BANDS = 16  # jobs the served image is split into (row bands)
BYTES_PER_STEP = 128  # algorithmic bytes per electron-step: a 64 B SoA record read and written


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if "Active" in v and "Not" not in v:
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def linescan_inputs(rank):
    from cudamonsel_b200 import replicas, scenes
    centers = scenes.linescan_pixels(NPIX, 1e-9, 0.0, -120e-9)
    return centers, replicas.pixel_keys(rank, NPIX)


# ------------------------------------------------------------------ CPU arms
def ref_binary():
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    data_ok = os.path.isdir(os.path.join(ROOT, "oracle", "_ref", "gov"))
    return exe if os.path.exists(exe) and data_ok else None


def cpu_sample(nproc, pixels_per_proc, nprim, seed):
    """Run the reference's compiled CPU code (or the oracle port) on nproc processes, each on its
    own pixels of the linescan; returns (primaries, seconds of the slowest transport loop, kind)."""
    from cudamonsel_b200 import data
    exe = ref_binary()
    x0 = -(NPIX - 1) / 2.0
    if exe:
        procs = []
        for p in range(nproc):
            start = x0 + (p * 37) % NPIX
            procs.append(subprocess.Popen([exe, "run2", str(nprim), str(seed + p), data.SI_TABLES, "%g" % start, "1",
                                           str(pixels_per_proc), "%g" % BEAM_EV], cwd=os.path.dirname(exe),
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
        secs = []
        for pr in procs:
            out, _ = pr.communicate()
            if pr.returncode != 0:
                raise RuntimeError("reference run failed")
            secs += [float(l.split()[1]) for l in out.splitlines() if l.startswith("seconds")]
        return nproc * pixels_per_proc * nprim, max(secs), "reference"
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    args = [(p, pixels_per_proc, nprim, seed) for p in range(nproc)]
    t0 = time.perf_counter()
    with ctx.Pool(nproc) as pool:
        pool.map(_oracle_worker, args)
    return nproc * pixels_per_proc * nprim, time.perf_counter() - t0, "port"


def _oracle_worker(a):
    p, npx, nprim, seed = a
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from cudamonsel_b200 import scenes
    sc = scenes.lines()
    centers = scenes.linescan_pixels(NPIX, 1e-9, 0.0, -120e-9)[(p * 37) % NPIX:][:npx]
    pyoracle.run_scene(sc, centers, 1e-9, scenes.eV(BEAM_EV), nprim, seed + p, NBINS)
    return 0


def reference_arm(a, rank):
    if rank != 0:
        return 0
    nproc = os.cpu_count() or 1
    for _ in range(a.warmup):
        cpu_sample(nproc, 1, 100, 7)
    prim = 0
    secs = 0.0
    kind = None
    for k in range(a.steps):
        n, s, kind = cpu_sample(nproc, 2, 250, 100 + k * nproc)
        prim += n
        secs += s
    v = prim / secs
    sample = "%d processes x 2 pixels x 250 primaries per step" % nproc
    line = {"metric": METRIC, "value": v, "unit": "primaries/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1000 * secs / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": sample}, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "primaries/s", "cores": nproc, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": "primaries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the served-stream latency measurement")
    ap.add_argument("--no-image", action="store_true", help="skip the rough-line image (FP32 vs FP64)")
    ap.add_argument("--no-deep", action="store_true", help="skip the 10 keV deep-penetration layout")
    ap.add_argument("--deep-side", type=int, default=128, help="pixels per side of the deep scan (full size 512)")
    ap.add_argument("--deep-primaries", type=int, default=250, help="primaries per pixel of the deep scan (full 500)")
    ap.add_argument("--serve-jobs", type=int, default=None, help="jobs in the served stream (full size 2000)")
    ap.add_argument("--serve-scale", type=float, default=None, help="size scale of the served jobs (full size 1)")
    ap.add_argument("--serve-rate", type=float, default=None, help="mean arrival rate of the served stream (1/s)")
    ap.add_argument("--no-autotune", action="store_true", help="run with the default launch settings")
    ap.add_argument("--profile-run", action="store_true",
                    help="run one FP32 step of the workload (host-driven replays) and exit: the case for ncu")
    ap.add_argument("--flight-units", type=int, nargs=2, metavar=("START", "END"),
                    help="print the electron-steps the flight kernel took in iterations [START, END) of the "
                         "--profile-run step (multiples of 16; two runs stopped by the iteration limit) and exit")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3) if a.impl == "ours" else a.warmup
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return reference_arm(a, rank)

    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from cudamonsel_b200 import capi, replicas, scenes
    from cudamonsel_b200 import stats as ystats

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    eng = capi.Engine(local)
    sc = scenes.lines()
    h = scenes.build_engine(sc, eng)
    centers, keys = linescan_inputs(rank)
    dev = torch.device("cuda", local)
    t_center = torch.tensor(centers.ravel(), dtype=torch.float64, device=dev)
    t_energy = torch.full((NPIX,), scenes.eV(BEAM_EV), dtype=torch.float64, device=dev)
    t_nprim = torch.full((NPIX,), NPRIM, dtype=torch.int32, device=dev)
    t_nbins = torch.full((NPIX,), NBINS, dtype=torch.int32, device=dev)
    t_keys = torch.tensor(keys.astype(np.int64), dtype=torch.int64, device=dev)
    stride = NBINS + 2
    t_back = torch.zeros((NPIX, stride), dtype=torch.int32, device=dev)
    t_fwd = torch.zeros((NPIX, stride), dtype=torch.int32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    stream = torch.cuda.current_stream(dev)
    import ctypes as C

    def desc(prec, profile=0):
        P = lambda t, ty: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ty))
        return capi.RunDesc(h["chamber"], prec, NPIX, 1e-9, P(t_center, C.c_double), P(t_energy, C.c_double),
                            P(t_nprim, C.c_int), P(t_nbins, C.c_int), 0, stride, 0, 0, P(t_keys, C.c_uint64), profile)

    def step(prec, profile=0):
        return eng.run_device(desc(prec, profile), t_back.data_ptr(), t_fwd.data_ptr(), stream.cuda_stream)

    prec = capi.PREC_FP32
    if a.flight_units:
        # the profiled replay stops at a multiple of 16 iterations when the limit is reached (CM_ELIMIT, stats
        # still written): the difference of two such runs is what the flight launches of the window took
        got = []
        for lim in a.flight_units:
            d = desc(prec, profile=1)
            d.max_iterations = lim
            st = capi.RunStats()
            eng.L.cm_run_device(eng.h, C.byref(d), C.c_void_p(t_back.data_ptr()), C.c_void_p(t_fwd.data_ptr()),
                                C.byref(st), C.c_void_p(stream.cuda_stream))
            torch.cuda.synchronize()
            got.append((int(st.iterations), int(st.units[0])))
        n = got[1][0] - got[0][0]
        print("flight electron-steps in iterations [%d, %d): %d (%.1f per launch)" % (
            got[0][0], got[1][0], got[1][1] - got[0][1], (got[1][1] - got[0][1]) / max(1, n)))
        eng.close()
        return 0
    if a.profile_run:
        # the host-driven replay of the same kernels (profile=1): ncu cannot profile the kernel nodes of
        # the device-driven loop's graph, whose WHILE loops are conditional nodes
        st = step(prec, profile=1)
        torch.cuda.synchronize()
        print("profile run: %d primaries, %d electron-steps, %d iterations" % (st.primaries, st.steps, st.iterations))
        eng.close()
        return 0
    # launch settings picked by the engine's autotuner on this workload (outside the timed region)
    tuned = {}
    if not a.no_autotune:
        for name, pr in (("fp32", capi.PREC_FP32), ("fp64", capi.PREC_FP64)):
            tt = eng.autotune(h["chamber"], centers, scenes.eV(BEAM_EV), NPRIM, NBINS, 1e-9, 0, precision=pr,
                              pixel_keys=keys)
            tuned[name] = {k: v for k, v in tt.as_dict().items() if k != "ms"}
    for _ in range(a.warmup):
        step(prec)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    stats = []
    torch.cuda.synchronize()
    for k in range(a.steps):
        flush.zero_()
        ev[k][0].record(stream)
        stats.append(step(prec))
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = replicas.max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in ev), dev)
    back32 = t_back.cpu().numpy().astype(np.int64)
    prim_per_rank = NPIX * NPRIM
    value = replicas.job_rate(prim_per_rank * a.steps, world, ms)

    # FP64 plain form on the same workload: throughput and the yield error of FP32 against it
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step(capi.PREC_FP64)  # untimed: builds the FP64 scene and wave buffers
    flush.zero_()
    e0.record(stream)
    st64 = step(capi.PREC_FP64)
    e1.record(stream)
    torch.cuda.synchronize()
    ms64 = e0.elapsed_time(e1)
    back64 = t_back.cpu().numpy().astype(np.int64)
    b32, s32 = scenes.yields(back32.sum(0), prim_per_rank, BEAM_EV, NBINS)
    b64, s64 = scenes.yields(back64.sum(0), prim_per_rank, BEAM_EV, NBINS)
    yerr = {"bse_fp32": float(b32[0]), "bse_fp64": float(b64[0]), "se_fp32": float(s32[0]), "se_fp64": float(s64[0]),
            "bse_rel_err": float(abs(b32[0] - b64[0]) / b64[0]), "se_rel_err": float(abs(s32[0] - s64[0]) / s64[0])}
    # per pixel: the FP32 yields against LB independent FP64 batches of LN primaries per pixel (streams of
    # their own), each pixel's variance from its batches; and the per-pixel difference from the FP64 run on
    # the same streams
    LB, LN = 8, 500
    fb, fs = [], []
    for r in range(LB):
        kb = keys + np.uint64((r + 1) * 1_000_000_007)
        bb, _, _ = eng.run(h["chamber"], centers, scenes.eV(BEAM_EV), LN, NBINS, 1e-9, 0, precision=capi.PREC_FP64,
                           pixel_keys=kb)
        yb = scenes.yields(bb, LN, BEAM_EV, NBINS)
        fb.append(yb[0])
        fs.append(yb[1])
    pb32, ps32 = scenes.yields(back32, NPRIM, BEAM_EV, NBINS)
    pb64, ps64 = scenes.yields(back64, NPRIM, BEAM_EV, NBINS)
    yerr["per_pixel"] = {
        "method": "FP32 run (2000/px) vs %d independent FP64 batches of %d/px; t per pixel as normal z" % (LB, LN),
        "bse": ystats.z_summary(ystats.scan_z(np.array(fb), LN, pb32, NPRIM)),
        "se": ystats.z_summary(ystats.scan_z(np.array(fs), LN, ps32, NPRIM)),
        "same_streams_abs_err": {"bse_mean": float(np.abs(pb32 - pb64).mean()),
                                 "bse_max": float(np.abs(pb32 - pb64).max()),
                                 "se_mean": float(np.abs(ps32 - ps64).mean()),
                                 "se_max": float(np.abs(ps32 - ps64).max())}}

    # end to end through the C ABI with host buffers: H2D of the pixel arrays, D2H of the tallies
    e2e_ms = 0.0
    for k in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.run(h["chamber"], centers, scenes.eV(BEAM_EV), NPRIM, NBINS, 1e-9, 0, precision=prec, pixel_keys=keys)
        e2e_ms += 1000 * (time.perf_counter() - t0)
    e2e_value = replicas.job_rate(prim_per_rank * a.steps, world, replicas.max_over_ranks(e2e_ms, dev))
    h2d = NPIX * (3 * 8 + 8 + 4 + 4 + 8)
    d2h = 2 * NPIX * stride * 4

    steps_total = sum(s.steps for s in stats)
    # the queue kernels, spawn and loop kernel of every iteration, the tail kernel, and the run's two gates
    launches = sum(sum(int(x) for x in s.kernel_launches) + int(s.step_launches) + 2 for s in stats)
    # roofline of the dominant kernel: one more step of the same workload with CUDA events
    # between the kernels of every iteration (event nodes inside the captured graphs); the tail
    # iterations run k_steps ("steps" in the shares), the others the six queue kernels
    flush.zero_()
    prof = [step(prec, profile=1)]
    torch.cuda.synchronize()
    kms = np.zeros(6)
    units = np.zeros(4)
    step_ms = 0.0
    for s in prof:
        kms += np.array(list(s.kernel_ms))
        units += np.array(list(s.units))
        step_ms += s.step_ms
    names = capi.RunStats.KERNELS
    dom = int(np.argmax(kms[:4]))
    nlaunch = sum(int(s.kernel_launches[dom]) for s in prof)
    per_launch_units = units[dom] / max(1, nlaunch)
    avg_ms = kms[dom] / max(1, nlaunch)
    achieved = units[dom] * BYTES_PER_STEP / (kms[dom] / 1000.0) / 1e9
    peak, peak_kind = peaks()
    # DRAM traffic of the dominant kernel: bytes per electron-step from an ncu capture of three heavy launches
    # of this workload (profiles/traffic.json), scaled to this run's mean electron-steps per launch
    traffic = None
    issue = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        per = json.load(open(tf)).get(names[dom])
        if isinstance(per, dict) and per.get("bytes_per_unit"):
            traffic = float(per["bytes_per_unit"]) * per_launch_units
        if isinstance(per, dict) and per.get("warp_instructions_per_unit"):
            # the kernel is issue- and latency-bound: its instruction rate against the SMs' issue peak (4 warp
            # schedulers per SM, one instruction per cycle each, at the SM clock sampled during the timed steps)
            issue = {"warp_instructions_per_unit": per["warp_instructions_per_unit"], "sm_count": 148,
                     "schedulers_per_sm": 4}

    # batched image: rough lines (3 x 128 segments), 256 x 256 pixels at 2 nm, Poisson(300) primaries per
    # pixel, energy per row from {300, 500, 1000} eV; FP32 batched form against the FP64 plain form
    image_line = None
    if not a.no_image:
        img = scenes.rough_lines(seed=0)
        eimg = capi.Engine(local)
        hi = scenes.build_engine(img, eimg)
        ic, ie, inp, inb = scenes.rough_image(seed=rank)
        ikeys = np.arange(len(ic), dtype=np.uint64) + np.uint64(7_000_003 * (rank + 1))
        # both precisions autotuned on the first eighth of the pixel rows (outside the timed runs).  The FP32
        # batched form runs with its tuned settings; the plain FP64 form, the target's comparison, with the
        # default launch settings; FP64 with its own tuned settings is timed once more for the stricter ratio.
        itune = {}
        if not a.no_autotune:
            band = slice(0, len(ic) // 8)
            for name, pr in (("fp32", capi.PREC_FP32), ("fp64", capi.PREC_FP64)):
                tt = eimg.autotune(hi["chamber"], ic[band], ie[band], inp[band], inb[band], 1e-9, 0, precision=pr,
                                   pixel_keys=ikeys[band])
                itune[name] = {k: v for k, v in tt.as_dict().items() if k != "ms"}
            eimg.set_tuning(capi.PREC_FP64)  # the plain form: default settings
        # IMAGE_REPEATS runs per precision, each on streams of its own: throughput as the median with its
        # spread, yields compared per pixel (pooled t over the repeats) and over the image
        reps = {"fp32": [], "fp64": []}
        ys = {"fp32": [], "fp64": []}
        e_eV = ie / scenes.EV
        first32 = None
        for r in range(IMAGE_REPEATS):
            for q, (name, pr) in enumerate((("fp32", capi.PREC_FP32), ("fp64", capi.PREC_FP64))):
                kr = ikeys + np.uint64((2 * r + q + 1) * 1_000_000_007)
                t0 = time.perf_counter()
                ib, _, ist = eimg.run(hi["chamber"], ic, ie, inp, inb, 1e-9, 0, precision=pr, pixel_keys=kr)
                reps[name].append((ist.device_ms, time.perf_counter() - t0, int(ist.steps)))
                ys[name].append(scenes.yields(ib.astype(np.int64), np.maximum(inp, 1), e_eV, inb))
                if first32 is None and name == "fp32":
                    first32 = (ib, kr)
        fp64_tuned = None
        if "fp64" in itune:
            t = itune["fp64"]
            eimg.set_tuning(capi.PREC_FP64, t["wave"], t["tail_below"], t["tail_steps"], t["blocks_per_sm"], t["pool"])
            _, _, tst = eimg.run(hi["chamber"], ic, ie, inp, inb, 1e-9, 0, precision=capi.PREC_FP64,
                                 pixel_keys=ikeys + np.uint64(99 * 1_000_000_007))
            fp64_tuned = int(inp.sum()) / (tst.device_ms / 1e3)
        # The same image served: IMAGE_BANDS row bands submitted at once to the job server (continuous
        # batching, FP32, the batched form's tuned settings); primaries/s over the makespan against the FP64
        # plain form's rate above, and each band's tallies against the batched FP32 run on the same streams
        served = None
        if not a.no_serving:
            srv = capi.Server(local, IMAGE_BANDS, SERVE_BUDGET_GB)
            if "fp32" in itune:
                t = itune["fp32"]
                srv.tune(capi.PREC_FP32, t["wave"], t["tail_below"], t["tail_steps"], t["blocks_per_sm"], t["pool"])
            rows = np.array_split(np.arange(len(ic)), IMAGE_BANDS)
            jobs = [srv.submit(eimg, hi["chamber"], ic[b], ie[b], inp[b], inb[b], 1e-9, 0, capi.PREC_FP32,
                               pixel_keys=first32[1][b]) for b in rows]
            infos = [srv.wait(j) for j in jobs]
            outs = [srv.result(j) for j in jobs]
            srv.close()
            same = all(np.array_equal(o[0], first32[0][b][:, :o[0].shape[1]]) and
                       not first32[0][b][:, o[0].shape[1]:].any() for o, b in zip(outs, rows))
            mk = max(i.end_s for i in infos) - min(i.submit_s for i in infos)
            lat = np.array([i.end_s - i.submit_s for i in infos])
            served = {"bands": IMAGE_BANDS, "primaries_per_s": int(inp.sum()) / mk, "makespan_s": mk,
                      "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                      "tallies_equal_batched": bool(same)}
        eimg.close()
        ntot = int(inp.sum())
        rate = {k: [ntot / (m / 1e3) for m, _, _ in v] for k, v in reps.items()}
        err = {}
        for j, nm in ((0, "bse"), (1, "se")):
            m32 = [(y[j] * inp).sum() / ntot for y in ys["fp32"]]
            m64 = [(y[j] * inp).sum() / ntot for y in ys["fp64"]]
            z, a32, a64, se = ystats.pooled_z(m32, m64)
            err[nm + "_fp32"], err[nm + "_fp64"], err[nm + "_rel_err"] = a32, a64, abs(a32 - a64) / a64
            err[nm + "_image_z"] = z
            err[nm + "_per_pixel"] = ystats.z_summary(ystats.repeats_z(
                [y[j] for y in ys["fp32"]], [y[j] for y in ys["fp64"]], nprim=np.maximum(inp, 1), groups=ie))
        err["per_pixel_method"] = ("%d FP32 vs %d FP64 repeats on streams of their own; each pixel's variance "
                                   "v(yield)/nprim, v pooled over the pixels of the same beam energy and mean-yield "
                                   "quantile (32 bins)" % (IMAGE_REPEATS, IMAGE_REPEATS))
        image_line = {"workload": "rough lines 3 x 128 segments (sidewall offsets N(0, 1.5 nm)), 256 x 256 px at "
                                  "2 nm, Poisson(300)/px, E per row in {300, 500, 1000} eV",
                      "primaries": ntot, "tuning": itune or "defaults", "repeats": IMAGE_REPEATS,
                      "fp32_primaries_per_s": statistics.median(rate["fp32"]),
                      "fp64_primaries_per_s": statistics.median(rate["fp64"]),
                      "fp32_primaries_per_s_range": [min(rate["fp32"]), max(rate["fp32"])],
                      "fp64_primaries_per_s_range": [min(rate["fp64"]), max(rate["fp64"])],
                      "fp64_settings": "defaults (the plain form)",
                      "fp32_over_fp64": statistics.median(rate["fp32"]) / statistics.median(rate["fp64"]),
                      "fp32_over_fp64_worst": min(rate["fp32"]) / max(rate["fp64"]),
                      "fp64_tuned_primaries_per_s": fp64_tuned,
                      "fp32_over_fp64_tuned": (statistics.median(rate["fp32"]) / fp64_tuned) if fp64_tuned else None,
                      "fp32_e2e_s": statistics.median(v[1] for v in reps["fp32"]),
                      "fp64_e2e_s": statistics.median(v[1] for v in reps["fp64"]),
                      "electron_steps_fp32": reps["fp32"][0][2],
                      "yield_error_vs_fp64": err}
        if served:
            served["fp32_served_over_fp64"] = served["primaries_per_s"] / statistics.median(rate["fp64"])
            image_line["served_fp32"] = served

    # deep penetration: 16 x 16 seed-placed blocks and cylinders (PMMA or Si, 20-300 nm) on Si, 10 keV, a
    # --deep-side^2 scan over the 5.12 um layout, --deep-primaries per pixel, FP32 against FP64; the
    # roofline of its dominant kernel from a profiled FP32 run of every second row and column
    deep_line = None
    if not a.no_deep:
        dsc, dtop = scenes.deep_features(seed=0)
        edeep = capi.Engine(local)
        hd = scenes.build_engine(dsc, edeep)
        side, dprim = a.deep_side, a.deep_primaries
        step_m = 5.12e-6 / side
        xs = (np.arange(side) - (side - 1) / 2.0) * step_m
        gx, gy = np.meshgrid(xs, xs)
        dc = np.stack([gx.ravel(), gy.ravel(), np.full(side * side, -(dtop + 20e-9))], axis=1)
        dkeys = np.arange(side * side, dtype=np.uint64) + np.uint64(5_000_011 * (rank + 1))
        druns = {}
        for name, pr in (("fp32", capi.PREC_FP32), ("fp64", capi.PREC_FP64)):
            db, _, dst = edeep.run(hd["chamber"], dc, scenes.eV(10000.0), dprim, 1000, 1e-9, 0, precision=pr,
                                   pixel_keys=dkeys)
            druns[name] = (db, dst)
        sub = (np.arange(side)[:, None] % 2 == 0) & (np.arange(side)[None, :] % 2 == 0)
        sub = sub.ravel()
        _, _, pst = edeep.run(hd["chamber"], dc[sub], scenes.eV(10000.0), dprim, 1000, 1e-9, 0,
                              precision=capi.PREC_FP32, pixel_keys=dkeys[sub], profile=1)
        edeep.close()
        dk = int(np.argmax(list(pst.kernel_ms)[:4]))
        dach = pst.units[dk] * BYTES_PER_STEP / (pst.kernel_ms[dk] / 1000.0) / 1e9
        y32 = scenes.yields(druns["fp32"][0].astype(np.int64), dprim, 10000.0, 1000)
        y64 = scenes.yields(druns["fp64"][0].astype(np.int64), dprim, 10000.0, 1000)
        nd = side * side * dprim
        deep_line = {"workload": "16 x 16 blocks/cylinders (PMMA or Si, 20-300 nm) on Si, 10 keV, %d x %d px at "
                                 "%.0f nm, %d primaries/px" % (side, side, step_m * 1e9, dprim), "primaries": nd,
                     "fp32_primaries_per_s": nd / (druns["fp32"][1].device_ms / 1e3),
                     "fp64_primaries_per_s": nd / (druns["fp64"][1].device_ms / 1e3),
                     "fp32_over_fp64": druns["fp64"][1].device_ms / druns["fp32"][1].device_ms,
                     "electron_steps_fp32": int(druns["fp32"][1].steps),
                     "electron_steps_per_s_fp32": druns["fp32"][1].steps / (druns["fp32"][1].device_ms / 1e3),
                     "roofline": {"bound": "hbm", "kernel": names[dk], "achieved": dach, "peak": peak,
                                  "unit": "GB/s", "frac": dach / peak, "peak_kind": peak_kind,
                                  "sample": "profiled FP32 run of every 2nd row and column",
                                  "kernel_ms_share": dict({n: float(v / (sum(pst.kernel_ms) + pst.step_ms))
                                                           for n, v in zip(names, pst.kernel_ms)},
                                                          steps=float(pst.step_ms / (sum(pst.kernel_ms) + pst.step_ms)))},
                     "yield_error_map_vs_fp64": {
                         "bse_mean_abs": float(np.abs(y32[0] - y64[0]).mean()),
                         "bse_max_abs": float(np.abs(y32[0] - y64[0]).max()),
                         "se_mean_abs": float(np.abs(y32[1] - y64[1]).mean()),
                         "se_max_abs": float(np.abs(y32[1] - y64[1]).max()),
                         "bse_image_mean_rel_err": float(abs(y32[0].mean() - y64[0].mean()) / y64[0].mean()),
                         "se_image_mean_rel_err": float(abs(y32[1].mean() - y64[1].mean()) / y64[1].mean()),
                         # at 10 keV the FP32 and FP64 trajectories decorrelate after a few hundred steps, so
                         # the difference is statistical: z = difference / combined standard error of the means
                         "bse_image_mean_z": float((y32[0].mean() - y64[0].mean()) / np.sqrt(
                             (y32[0].var(ddof=1) + y64[0].var(ddof=1)) / y32[0].size)),
                         "se_image_mean_z": float((y32[1].mean() - y64[1].mean()) / np.sqrt(
                             (y32[1].var(ddof=1) + y64[1].var(ddof=1)) / y32[1].size))}}

    # served stream: random scan jobs (1-8 lines/cylinders on Si, 200-5000 eV, images or linescans) at
    # Poisson arrivals through the job server, sizes scaled by SERVE_SCALE; p50/p99 of submit-to-done latency
    serving_line = None
    if not a.no_serving:
        from cudamonsel_b200 import serving
        njobs = a.serve_jobs or SERVE_JOBS
        sscale = a.serve_scale or SERVE_SCALE
        srate = a.serve_rate or SERVE_RATE
        js = serving.make_jobs(njobs, seed=100 + rank, scale=sscale)
        out = serving.serve(js, rate_per_s=srate, slots=SERVE_SLOTS, budget_gb=SERVE_BUDGET_GB, seed=200 + rank,
                            device=local)
        lat = out["latency"]
        # the same jobs submitted all at once (the server saturated), FP32 and FP64: served throughput
        sat = {}
        for name, pr in (("fp32", capi.PREC_FP32), ("fp64", capi.PREC_FP64)):
            o = serving.serve(js, rate_per_s=None, slots=SERVE_SLOTS, budget_gb=SERVE_BUDGET_GB, precision=pr,
                              device=local)
            sat[name] = {"primaries_per_s": o["primaries"] / o["makespan"],
                         "electron_steps_per_s": o["steps"] / o["makespan"], "makespan_s": o["makespan"],
                         "p50_s": float(np.percentile(o["latency"], 50)),
                         "p99_s": float(np.percentile(o["latency"], 99))}
        sat["fp32_over_fp64"] = sat["fp32"]["primaries_per_s"] / sat["fp64"]["primaries_per_s"]
        serving_line = {"jobs": njobs, "rate_per_s": srate, "slots": SERVE_SLOTS,
                        "budget_gb": SERVE_BUDGET_GB, "size_scale": sscale,
                        "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                        "makespan_s": out["makespan"], "primaries": out["primaries"],
                        "primaries_per_s": out["primaries"] / out["makespan"],
                        "electron_steps_per_s": out["steps"] / out["makespan"],
                        "saturated": sat}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        nproc = os.cpu_count() or 1
        n, secs, kind = cpu_sample(nproc, 4, 500, 1)
        cpu = {"value": n / secs, "unit": "primaries/s", "cores": nproc, "kind": kind,
               "sample": "%d processes x 4 linescan pixels x 500 primaries" % nproc}

    if issue and clk and clk.get("sm_mhz"):
        rate = units[dom] / (kms[dom] / 1000.0) * issue["warp_instructions_per_unit"]
        peak_issue = issue["sm_count"] * issue["schedulers_per_sm"] * clk["sm_mhz"] * 1e6
        issue.update({"achieved_warp_instructions_per_s": rate, "peak_warp_instructions_per_s": peak_issue,
                      "frac": rate / peak_issue})
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "primaries/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "pixels": NPIX, "primaries_per_pixel": NPRIM, "beam_eV": BEAM_EV,
                           "precision": "f32 transport, f64 positions and plane solves",
                           "l2": "flushed between steps (256 MB write)", "parallelism": "replicas x%d" % world,
                           "tuning": tuned or "defaults"},
                "electron_steps_per_s": world * steps_total / (ms / 1000.0),
                "fp64": {"value": prim_per_rank / (ms64 / 1000.0), "unit": "primaries/s", "steps": int(st64.steps)},
                "yield_error_vs_fp64": yerr,
                "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak,
                             "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "bytes_per_unit": BYTES_PER_STEP, "units_per_launch": per_launch_units,
                             "avg_launch_ms": avg_ms},
                "issue_roofline": issue,
                "kernel_ms_share": dict({n: float(v / (kms.sum() + step_ms)) for n, v in zip(names, kms)},
                                        steps=float(step_ms / (kms.sum() + step_ms))),
                "clocks": clk, "gpu_launches": launches,
                "e2e": {"value": e2e_value, "unit": "primaries/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h},
                "cpu_baseline": cpu, "serving": serving_line, "image": image_line, "deep": deep_line}
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
