// cm_server.cuh -- job server for streams of scan jobs (included by cm_engine.cu).
//
// Continuous batching: the jobs of one precision and set of run options share one wave of electrons on the
// GPU.  A batcher (one host thread, one engine context) merges the scene of every job it admits into one
// scene -- its chamber and regions appended unless an earlier job of the batch has the same geometry (then
// it shares that chamber), scattering tables, materials and scatter models shared with earlier jobs when
// their contents are equal -- and appends the job's pixels to the batch's pixel tables (with the job's
// chamber, beam width, tally row and job number per pixel).  A job's primaries join the wave as soon as
// those of the jobs admitted before it have all started, so new jobs fill the room the ending cascades of
// earlier ones leave; the wave does not drain between jobs.  Jobs are admitted first in, first out while
// fewer than `slots` are in the batch and their pixel and tally buffers fit `budget_gb`; a new batch first
// gathers the submissions of a burst, so that its scene is built once.  Per job the device counts the
// electrons alive and their steps; a job is done when its primaries have all started and none of its
// electrons is left, and its tallies are copied out.  A
// job's tallies depend only on its scene, pixels and stream keys: the same alone, in any mix and
// through cm_run.  Cancelling a running job stops its unstarted primaries; the ones in flight end
// on their own.
//
// The batcher replays captured rounds of transport iterations (the queue kernels while the wave is full,
// the several-steps kernel in the tail) and between rounds admits jobs, reads the counters and finishes
// jobs.  When the batch runs empty its scene and tables are dropped, so memory stays bounded.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

namespace cm {

struct JobRecord {
  int id = 0;
  int state = CM_JOB_QUEUED;
  int error = 0;
  std::string message;
  // the scene, copied from the submitting context
  int options = 0;
  std::map<int, HMott> mott;
  std::vector<HTable> tables;
  std::vector<HMaterial> mats;
  std::vector<HMsm> msms;
  std::vector<HShape> shapes;
  std::vector<HRegion> regions;
  // the run, with its host arrays copied
  cm_run_desc desc;
  std::vector<double> center, energy;
  std::vector<int> nprim, nbins;
  std::vector<uint64_t> keys;
  size_t footprint = 0;
  // results
  std::vector<uint32_t> back, fwd;
  cm_run_stats stats;
  double t_submit = 0, t_start = 0, t_end = 0;
  std::atomic<int> cancel{0};
  // place in the batch
  int slot = -1;                      // its counters in the batch
  unsigned long long g0 = 0, g1 = 0;  // its primaries in the batch's sequence of primaries
  size_t tally0 = 0;                  // its first tally element in the batch's tally arrays
  bool stop_sent = false;
};

// a device array that grows between rounds (the old contents are kept)
template <typename T> struct DevVec {
  T* p = nullptr;
  size_t cap = 0;
  int reserve(size_t n) {
    if (n <= cap) return 0;
    size_t c = cap ? cap : 1024;
    while (c < n) c *= 2;
    T* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, c * sizeof(T));
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      return fail(CM_ENOMEM, "job server: device memory exhausted growing the batch tables");
    }
    if (p) {
      CM_CUDA(cudaMemcpy(q, p, cap * sizeof(T), cudaMemcpyDeviceToDevice));
      cudaFree(p);
    }
    p = q;
    cap = c;
    return 0;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

static bool same_table(const HTable& a, const HTable& b) {
  if (a.dim != b.dim || a.role != b.role || a.v != b.v) return false;
  for (int k = 0; k < a.dim; ++k)
    if (a.n[k] != b.n[k] || a.x[k] != b.x[k]) return false;
  return true;
}
static bool same_material(const HMaterial& a, const HMaterial& b) {
  return a.Z == b.Z && a.A == b.A && a.wf == b.wf && a.core == b.core && a.density == b.density &&
         a.workfunction == b.workfunction && a.ecb == b.ecb && a.bandgap == b.bandgap;
}
static bool same_mech(const HMech& a, const HMech& b) {
  return a.kind == b.kind && a.method == b.method && a.energyOffset == b.energyOffset &&
         std::equal(a.tables, a.tables + 4, b.tables) && a.energySEgen == b.energySEgen && a.breakE == b.breakE &&
         a.ratemult == b.ratemult && a.phononE == b.phononE && a.temperature == b.temperature && a.eps0 == b.eps0 &&
         a.epsInf == b.epsInf && a.prefactor == b.prefactor && a.extinction == b.extinction;
}
static bool same_msm(const HMsm& a, const HMsm& b) {
  if (a.material != b.material || a.mechs.size() != b.mechs.size() || a.csd != b.csd || a.breakE != b.breakE ||
      a.minSet != b.minSet || a.minE != b.minE || a.classical != b.classical || a.lambda != b.lambda)
    return false;
  for (size_t k = 0; k < a.mechs.size(); ++k)
    if (!same_mech(a.mechs[k], b.mechs[k])) return false;
  return true;
}

// shape k of a job (its child indices moved by shape0) equals shape a of the batch's scene
static bool same_shape(const HShape& a, const HShape& k, int shape0) {
  if (a.kind != k.kind) return false;
  switch (k.kind) {
    case SHAPE_SPHERE:
      return std::equal(a.c, a.c + 3, k.c) && a.r == k.r;
    case SHAPE_PLANES:
      return a.n == k.n && a.p == k.p;
    case SHAPE_INTERSECTION:
    case SHAPE_UNION:
      return a.a == k.a + shape0 && a.b == k.b + shape0;
    case SHAPE_CYLINDER:
      return std::equal(a.e0, a.e0 + 3, k.e0) && std::equal(a.ax, a.ax + 3, k.ax) &&
             std::equal(a.nax, a.nax + 3, k.nax) && a.radius == k.radius && a.len2 == k.len2;
  }
  return false;
}

// Where a job's geometry sits in the batch's scene (merge_scene): jobs with the same geometry (a scan split
// into bands, repeated scans of one sample) share its chamber and regions.
struct MergedGeometry {
  int shape0, nshapes, region0, nregions;
};

static bool same_geometry(const cm_context* ctx, const MergedGeometry& g, const JobRecord& j,
                          const std::vector<int>& smap) {
  if (g.nshapes != (int)j.shapes.size() || g.nregions != (int)j.regions.size()) return false;
  for (int k = 0; k < g.nshapes; ++k)
    if (!same_shape(ctx->shapes[g.shape0 + k], j.shapes[k], g.shape0)) return false;
  for (int k = 0; k < g.nregions; ++k) {
    const HRegion& a = ctx->regions[g.region0 + k];
    const HRegion& r = j.regions[k];
    if (a.parent != (r.parent >= 0 ? r.parent + g.region0 : -1) || a.msm != smap[r.msm] ||
        a.shape != r.shape + g.shape0 || a.children.size() != r.children.size())
      return false;
    for (size_t c = 0; c < r.children.size(); ++c)
      if (a.children[c] != r.children[c] + g.region0) return false;
  }
  return true;
}

// the job's scene into the batch's scene: shared parts found by content, its shapes and regions appended
// unless a job before it in the batch had the same geometry; returns the job's chamber in the batch's scene
static int merge_scene(cm_context* ctx, std::vector<MergedGeometry>& merged, const JobRecord& j) {
  for (const auto& kv : j.mott)
    if (!ctx->mott.count(kv.first)) ctx->mott[kv.first] = kv.second;
  std::vector<int> tmap(j.tables.size()), mmap(j.mats.size()), smap(j.msms.size());
  for (size_t t = 0; t < j.tables.size(); ++t) {
    int hit = -1;
    for (size_t u = 0; u < ctx->tables.size() && hit < 0; ++u)
      if (same_table(ctx->tables[u], j.tables[t])) hit = (int)u;
    if (hit < 0) {
      hit = (int)ctx->tables.size();
      ctx->tables.push_back(j.tables[t]);
    }
    tmap[t] = hit;
  }
  for (size_t m = 0; m < j.mats.size(); ++m) {
    int hit = -1;
    for (size_t u = 0; u < ctx->mats.size() && hit < 0; ++u)
      if (same_material(ctx->mats[u], j.mats[m])) hit = (int)u;
    if (hit < 0) {
      hit = (int)ctx->mats.size();
      ctx->mats.push_back(j.mats[m]);
    }
    mmap[m] = hit;
  }
  for (size_t s = 0; s < j.msms.size(); ++s) {
    HMsm h = j.msms[s];
    h.material = mmap[h.material];
    for (HMech& k : h.mechs)
      if (k.kind == MECH_TABULATED)
        for (int q = 0; q < 4; ++q) k.tables[q] = tmap[k.tables[q]];
    int hit = -1;
    for (size_t u = 0; u < ctx->msms.size() && hit < 0; ++u)
      if (same_msm(ctx->msms[u], h)) hit = (int)u;
    if (hit < 0) {
      hit = (int)ctx->msms.size();
      ctx->msms.push_back(h);
    }
    smap[s] = hit;
  }
  for (const MergedGeometry& g : merged)
    if (same_geometry(ctx, g, j, smap)) return g.region0 + j.desc.chamber;  // the scene is unchanged
  const int shape0 = (int)ctx->shapes.size(), region0 = (int)ctx->regions.size();
  merged.push_back(MergedGeometry{shape0, (int)j.shapes.size(), region0, (int)j.regions.size()});
  for (HShape s : j.shapes) {
    if (s.kind == SHAPE_INTERSECTION || s.kind == SHAPE_UNION) {
      s.a += shape0;
      s.b += shape0;
    }
    ctx->shapes.push_back(s);
  }
  for (HRegion r : j.regions) {
    if (r.parent >= 0) r.parent += region0;
    r.msm = smap[r.msm];
    r.shape += shape0;
    for (int& c : r.children) c += region0;
    ctx->regions.push_back(r);
  }
  ctx->dirty();
  return region0 + j.desc.chamber;
}

// the jobs of one precision and run options in one shared wave
struct Batcher {
  int precision = CM_PREC_FP32, options = 0;
  cm_context* ctx = nullptr;
  std::thread thread;
  // the batch's pixel tables, tallies and job counters (grown as jobs join, kept until the batch empties)
  DevVec<double> pc, pe0, pe0ref, pwidth;
  DevVec<int> pnbins, pchamber, pjob, job_stop;
  DevVec<unsigned long long> prefix, pkey, ptally, job_alive, job_steps;
  DevVec<uint32_t> back, fwd;
  int npix = 0, slots = 0;
  unsigned long long total = 0;
  size_t tally_used = 0;
  bool counters_live = false;  // the device counters describe the current batch
  int pool_want = 0;           // secondary-pool records to ask for (doubled after an overflow)
  double emax_eV = 0;          // highest beam energy of the batch's jobs
  int restarts = 0;            // restarts of the current batch after overflows
  std::vector<MergedGeometry> merged;  // the geometries merged into the batch's scene
  bool waiting = false;        // jobs of this batcher wait in the queue (set before each round)
  std::vector<JobRecord*> active;
  // captured rounds of iterations for the current scene build and run buffers
  cudaGraphExec_t round_exec[2] = {nullptr, nullptr};
  cudaGraph_t round_graph[2] = {nullptr, nullptr};
  LoopKey round_key{};
  const void* round_buffers = nullptr;
  int round_pool = 0;
  void drop_rounds() {
    for (int k = 0; k < 2; ++k) {
      if (round_exec[k]) cudaGraphExecDestroy(round_exec[k]);
      if (round_graph[k]) cudaGraphDestroy(round_graph[k]);
      round_exec[k] = nullptr;
      round_graph[k] = nullptr;
    }
  }
  void release() {
    drop_rounds();
    DevVec<double>* d[] = {&pc, &pe0, &pe0ref, &pwidth};
    for (auto* x : d) x->release();
    DevVec<int>* i[] = {&pnbins, &pchamber, &pjob, &job_stop};
    for (auto* x : i) x->release();
    DevVec<unsigned long long>* u[] = {&prefix, &pkey, &ptally, &job_alive, &job_steps};
    for (auto* x : u) x->release();
    back.release();
    fwd.release();
  }
};

}  // namespace cm

struct cm_server {
  int device = 0;
  int max_active = 4;  // jobs in one batch at once
  size_t budget = 0;   // bytes the admitted jobs' own buffers may take
  size_t in_use = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<int> queue;  // admission order
  std::map<int, std::unique_ptr<cm::JobRecord>> jobs;
  std::map<std::pair<int, int>, std::unique_ptr<cm::Batcher>> batchers;  // by (precision, options)
  cm_tuning tune[2] = {};                                                 // per precision, for new batches
  int next_id = 0;
  bool stop = false;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace cm {

// device bytes a job needs in the batch: its pixel tables and tally rows
static size_t job_footprint(const cm_run_desc& d) {
  return (size_t)d.npix * (3 * 8 + 8 + 8 + 8 + 8 + 8 + 8 + 4 + 4 + 4) + 2 * (size_t)d.npix * d.hist_stride * 4 + 4096;
}

static void fill_info(const JobRecord& j, cm_job_info* info) {
  info->state = j.state;
  info->error = j.error;
  info->submit_s = j.t_submit;
  info->start_s = j.t_start;
  info->end_s = j.t_end;
  info->primaries = j.state == CM_JOB_DONE ? j.stats.primaries : 0;
  info->steps = j.state == CM_JOB_DONE ? j.stats.steps : 0;
}

// append one job to the batch: scene, pixel tables, tally rows, counters (between rounds, device idle)
static int batch_add(Batcher& b, JobRecord& j) {
  NvtxRange range("cm job admit");
  cm_context* ctx = b.ctx;
  const cm_run_desc& d = j.desc;
  PixelPrep p;
  int rc = prep_pixels(&d, j.center.data(), j.energy.data(), j.nprim.data(), j.nbins.data(), d.hist_stride, p);
  if (rc) return rc;
  const int n = d.npix;
  const size_t rows = (size_t)n * d.hist_stride;
  const size_t np = (size_t)b.npix + n;
  if ((rc = b.pc.reserve(3 * np)) || (rc = b.pe0.reserve(np)) || (rc = b.pe0ref.reserve(np)) ||
      (rc = b.pwidth.reserve(np)) || (rc = b.pnbins.reserve(np)) || (rc = b.pchamber.reserve(np)) ||
      (rc = b.pjob.reserve(np)) || (rc = b.prefix.reserve(np + 1)) || (rc = b.pkey.reserve(np)) ||
      (rc = b.ptally.reserve(np)) || (rc = b.back.reserve(b.tally_used + rows)) ||
      (rc = b.fwd.reserve(b.tally_used + rows)) || (rc = b.job_alive.reserve(b.slots + 1)) ||
      (rc = b.job_steps.reserve(b.slots + 1)) || (rc = b.job_stop.reserve(b.slots + 1)))
    return rc;
  const int chamber = merge_scene(ctx, b.merged, j);
  for (double e : p.e0) b.emax_eV = std::max(b.emax_eV, e);
  j.slot = b.slots++;
  j.g0 = b.total;
  j.g1 = b.total + p.total;
  j.tally0 = b.tally_used;
  std::vector<unsigned long long> prefix(n), ptally(n);
  for (int i = 0; i < n; ++i) {
    prefix[i] = b.total + p.prefix[i + 1];  // the batch's prefix entry after its pixel b.npix + i
    ptally[i] = b.tally_used + (size_t)i * d.hist_stride;
  }
  const std::vector<double> width(n, d.beam_width * 1e9);
  const std::vector<int> chambers(n, chamber), jobs(n, j.slot);
  const unsigned long long zero = 0;
  const int nostop = 0;
  cudaStream_t s = ctx->stream;
  if (b.npix == 0) CM_CUDA(cudaMemcpyAsync(b.prefix.p, &zero, 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.pc.p + 3 * (size_t)b.npix, p.center_nm.data(), 3 * (size_t)n * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.pe0.p + b.npix, p.e0.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.pe0ref.p + b.npix, p.e0ref.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.pwidth.p + b.npix, width.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.pnbins.p + b.npix, j.nbins.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.pchamber.p + b.npix, chambers.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.pjob.p + b.npix, jobs.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.prefix.p + b.npix + 1, prefix.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.pkey.p + b.npix, p.key.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.ptally.p + b.npix, ptally.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemsetAsync(b.back.p + b.tally_used, 0, rows * 4, s));
  CM_CUDA(cudaMemsetAsync(b.fwd.p + b.tally_used, 0, rows * 4, s));
  CM_CUDA(cudaMemcpyAsync(b.job_alive.p + j.slot, &zero, 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.job_steps.p + j.slot, &zero, 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.job_stop.p + j.slot, &nostop, 4, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaStreamSynchronize(s));  // the host vectors above end here
  b.npix += n;
  b.total = j.g1;
  b.tally_used += rows;
  return 0;
}

// rounds a batch runs between two reads of its counters while its wave is full and no job waits
constexpr int kRoundRepeats = 4;

// one round of the batch: kLoopBody iterations of the queue kernels, or of the tail kernels once every
// primary has started and fewer electrons are left than the tail threshold
template <typename R>
static int batch_round(Batcher& b) {
  NvtxRange range("cm server round");
  cm_context* ctx = b.ctx;
  DevScene<R>& ds = scene_of<R>(ctx);
  int rc;
  if ((rc = build_scene<R>(ctx, ds))) return rc;
  const cm_tuning tu = resolved_tuning<R>(ctx);
  const int W = tu.wave;
  RunBuffers<R>& rb0 = buffers_of<R>(ctx);
  if (b.counters_live) {
    // within a batch the buffers hold its electrons: they stay as they are (the launch settings and the
    // pool are chosen when the batch starts; an overflow restarts the batch with a larger pool)
    if (rb0.cap != W) return fail(CM_ESTATE, "job server: run buffers changed within a batch");
  } else {
    const int poolWant = std::max({pool_records(W, b.emax_eV, tu.pool), b.pool_want, rb0.cap == W ? rb0.poolCap : 0});
    if ((rc = ensure_buffers<R>(ctx, W, poolWant))) {
      if (rc != CM_ENOMEM || poolWant <= 8 * W || (rc = ensure_buffers<R>(ctx, W, 8 * W))) return rc;
    }
  }
  RunBuffers<R>& rb = buffers_of<R>(ctx);
  cudaStream_t s = ctx->stream;
  RunView<R> v;
#ifdef CM_TRACE
  v.trace = nullptr;
  v.ntrace = nullptr;
  v.tracecap = 0;
#endif
  v.s = ds.view;
  v.s.chamber = 0;  // each pixel names its own chamber
  v.w[0] = rb.w[0];
  v.w[1] = rb.w[1];
  v.pool = rb.pool;
  for (int k = 0; k < 3; ++k) v.q[k] = rb.q[k];
  v.c = ctx->counters;
  v.W = W;
  v.poolCap = rb.poolCap;
  v.io = rb.io;
  RunIO& io = *ctx->io_host;
  memset(&io, 0, sizeof(io));
  io.pc = b.pc.p;
  io.pe0 = b.pe0.p;
  io.pe0ref = b.pe0ref.p;
  io.pnbins = b.pnbins.p;
  io.prefix = b.prefix.p;
  io.pkey = b.pkey.p;
  io.npix = b.npix;
  io.back = b.back.p;
  io.fwd = b.fwd.p;
  io.pchamber = b.pchamber.p;
  io.pwidth = b.pwidth.p;
  io.ptally = b.ptally.p;
  io.pjob = b.pjob.p;
  io.job_alive = b.job_alive.p;
  io.job_steps = b.job_steps.p;
  io.job_stop = b.job_stop.p;
  CM_CUDA(cudaMemcpyAsync(rb.io, &io, sizeof(RunIO), cudaMemcpyHostToDevice, s));
  // the counters: started afresh for a new batch, else extended by the primaries of the jobs just added
  Counters& hc = *ctx->counters_host;
  if (!b.counters_live) {
    memset(&hc, 0, sizeof(hc));
    b.counters_live = true;
  }
  if (hc.total_primaries != b.total) {
    hc.total_primaries = b.total;
    hc.done = 0;
  }
  // several whole steps per thread (the tail kernels) whenever fewer electrons are in the wave and pool than
  // fill the GPU, even with primaries still to start; the refill then fills the wave only up to that many,
  // so a light load runs at the latency of a job alone and a heavy one through the queue kernels
  const long long left = (long long)hc.n[0] + hc.n[1] + std::min(hc.pool, v.poolCap);
  const bool tail = !(ctx->options & CM_OPT_QUEUE_STEPS) && left < tu.tail_below;
  hc.fill = tail ? std::min(W, tu.tail_below) : 0;
  CM_CUDA(cudaMemcpyAsync(ctx->counters, &hc, sizeof(Counters), cudaMemcpyHostToDevice, s));
  const int grid = ctx->nsm * tu.blocks_per_sm;
  v.s.nstaged = 0;
  RunView<R> vs = v;
  if (!(ctx->options & CM_OPT_GLOBAL_TABLES)) vs.s.nstaged = v.s.nstage;
  const size_t smem = (size_t)vs.s.nstaged * sizeof(R);
  const LoopKey key{ds.gen, 0, grid, ctx->nsm * CM_INEL_BLOCKS_PER_SM, tu.tail_steps, (int)vs.s.nstaged};
  if (!b.round_exec[0] || !(b.round_key == key) || b.round_buffers != (const void*)rb.w[0].px ||
      b.round_pool != rb.poolCap) {
    b.drop_rounds();
    for (int loop = 0; loop < 2; ++loop) {
      CM_CUDA(cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal));
      for (int it = 0; it < kLoopBody; ++it) {
        if (loop == 0) launch_queue_iteration<R>(ctx, v, vs, it & 1, grid, smem, ctx->cap_stream, nullptr, nullptr);
        else launch_tail_iteration<R>(v, vs, it & 1, grid, tu.tail_steps, smem, ctx->cap_stream, nullptr, nullptr);
      }
      CM_CUDA(cudaStreamEndCapture(ctx->cap_stream, &b.round_graph[loop]));
      CM_CUDA(cudaGraphInstantiate(&b.round_exec[loop], b.round_graph[loop], 0));
    }
    b.round_key = key;
    b.round_buffers = (const void*)rb.w[0].px;
    b.round_pool = rb.poolCap;
  }
  // While the wave is full and no job waits for admission, kRoundRepeats rounds run back to back before
  // the counters are read: the host's turn between rounds (counter copies, job bookkeeping) leaves the GPU
  // idle.  In the tail, where jobs end, and while jobs wait, one round per turn keeps latency short.
  const int reps = (!tail && !b.waiting) ? kRoundRepeats : 1;
  for (int r = 0; r < reps; ++r) CM_CUDA(cudaGraphLaunch(b.round_exec[tail ? 1 : 0], s));
  CM_CUDA(cudaMemcpyAsync(&hc, ctx->counters, sizeof(Counters), cudaMemcpyDeviceToHost, s));
  CM_CUDA(cudaStreamSynchronize(s));
  return 0;
}

// the jobs whose primaries have all started and whose electrons have all ended: tallies copied out;
// the jobs cancelled since the last round: their unstarted primaries stopped
static int batch_collect(Batcher& b, std::vector<JobRecord*>& finished) {
  NvtxRange range("cm job results");
  if (b.slots == 0 || !b.counters_live) return 0;
  const Counters& hc = *b.ctx->counters_host;
  std::vector<unsigned long long> alive(b.slots), steps(b.slots);
  CM_CUDA(cudaMemcpy(alive.data(), b.job_alive.p, (size_t)b.slots * 8, cudaMemcpyDeviceToHost));
  CM_CUDA(cudaMemcpy(steps.data(), b.job_steps.p, (size_t)b.slots * 8, cudaMemcpyDeviceToHost));
  for (size_t k = 0; k < b.active.size(); ++k) {
    JobRecord& j = *b.active[k];
    if (j.cancel.load() && !j.stop_sent) {
      const int one = 1;
      CM_CUDA(cudaMemcpy(b.job_stop.p + j.slot, &one, 4, cudaMemcpyHostToDevice));
      j.stop_sent = true;
    }
    if (hc.next_primary < j.g1 || alive[j.slot] != 0) continue;
    const size_t rows = (size_t)j.desc.npix * j.desc.hist_stride;
    j.back.resize(rows);
    j.fwd.resize(rows);
    CM_CUDA(cudaMemcpy(j.back.data(), b.back.p + j.tally0, rows * 4, cudaMemcpyDeviceToHost));
    CM_CUDA(cudaMemcpy(j.fwd.data(), b.fwd.p + j.tally0, rows * 4, cudaMemcpyDeviceToHost));
    memset(&j.stats, 0, sizeof(j.stats));
    j.stats.primaries = (int64_t)(j.g1 - j.g0);
    j.stats.steps = (int64_t)steps[j.slot];
    finished.push_back(&j);
    b.active.erase(b.active.begin() + k--);
  }
  return 0;
}

static void batch_reset(Batcher& b);

// The batch overflowed its secondary pool (a secondary was lost, so its tallies are void).  Every electron's
// random stream is keyed by its lineage, so the batch's jobs are run again from their start with twice the
// pool and give the tallies an unbounded pool would have given.
static int batch_restart(Batcher& b) {
  if (2LL * std::max(b.pool_want, b.round_pool) > (1LL << 30))
    return fail(CM_EOVERFLOW, "job server: secondary pool overflow with a pool of 2^30 records");
  b.pool_want = 2 * std::max(b.pool_want, b.round_pool);
  const std::vector<JobRecord*> again = b.active;
  batch_reset(b);
  ++b.restarts;
  b.active = again;  // a job that cannot be added again fails with the batch
  for (JobRecord* j : again) {
    j->stop_sent = false;
    const int rc = batch_add(b, *j);
    if (rc) return rc;
  }
  return 0;
}

// the batch ran empty: its scene and tables are dropped
static void batch_reset(Batcher& b) {
  cm_context_reset(b.ctx);
  b.merged.clear();
  b.ctx->options = b.options;
  b.npix = 0;
  b.slots = 0;
  b.total = 0;
  b.tally_used = 0;
  b.emax_eV = 0;
  b.counters_live = false;
  b.drop_rounds();
}

// submissions closer together than this (ms) are gathered into a new batch, for at most kGatherMaxMs
constexpr int kGatherMs = 5;
constexpr int kGatherMaxMs = 50;

template <typename R>
static void batcher_worker(cm_server* srv, Batcher* b) {
  cudaSetDevice(srv->device);
  for (;;) {
    std::vector<JobRecord*> admitted;
    {
      std::unique_lock<std::mutex> lk(srv->mu);
      auto mine = [&](const JobRecord& j) { return j.desc.precision == b->precision && j.options == b->options; };
      auto head_fits = [&]() {  // the first queued job of this batcher has room in the batch and the budget
        for (int id : srv->queue) {
          const JobRecord& j = *srv->jobs[id];
          if (!mine(j)) continue;
          return (int)b->active.size() < srv->max_active &&
                 (srv->in_use == 0 || srv->in_use + j.footprint <= srv->budget);
        }
        return false;
      };
      if (b->active.empty()) {
        srv->cv_work.wait(lk, [&] { return srv->stop || head_fits(); });
        // A new batch: jobs submitted together (a scan split into bands, a burst of requests) join it at
        // once, so that its scene is merged, uploaded and its rounds captured once rather than once per
        // job as they come in: admission waits while submissions keep arriving less than kGatherMs
        // apart, at most kGatherMaxMs.
        const auto t0 = std::chrono::steady_clock::now();
        while (!srv->stop && std::chrono::steady_clock::now() - t0 < std::chrono::milliseconds(kGatherMaxMs)) {
          const size_t q = srv->queue.size();
          if (!srv->cv_work.wait_for(lk, std::chrono::milliseconds(kGatherMs),
                                     [&] { return srv->stop || srv->queue.size() != q; }))
            break;
        }
      }
      if (srv->stop) return;
      while (head_fits()) {
        auto it = srv->queue.begin();
        while (!mine(*srv->jobs[*it])) ++it;
        JobRecord* j = srv->jobs[*it].get();
        srv->queue.erase(it);
        srv->in_use += j->footprint;
        j->state = CM_JOB_RUNNING;
        j->t_start = srv->now();
        admitted.push_back(j);
      }
    }
    int rc = 0;
    if (b->slots == 0 && !admitted.empty()) {  // a new batch takes the server's current launch settings
      std::lock_guard<std::mutex> lk(srv->mu);
      b->ctx->tune[b->precision] = srv->tune[b->precision];
    }
    std::vector<JobRecord*> added;
    for (JobRecord* j : admitted) {
      if (rc == 0) rc = batch_add(*b, *j);
      if (rc == 0) {
        b->active.push_back(j);
        added.push_back(j);
      }
    }
    std::vector<JobRecord*> finished;
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      b->waiting = false;
      for (int id : srv->queue)
        if (srv->jobs[id]->desc.precision == b->precision && srv->jobs[id]->options == b->options) {
          b->waiting = true;
          break;
        }
    }
    if (rc == 0 && !b->active.empty())
      rc = b->precision == CM_PREC_FP64 ? batch_round<double>(*b) : batch_round<float>(*b);
    if (rc == 0 && b->ctx->counters_host->error) rc = run_error(b->ctx->counters_host->error, *b->ctx->counters_host);
    if (rc == CM_EOVERFLOW) rc = batch_restart(*b);
    if (rc == 0) rc = batch_collect(*b, finished);
    const std::string msg = rc ? cm_last_error() : "";
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      const double t = srv->now();
      for (JobRecord* j : finished) {
        j->stats.pool_restarts = b->restarts;
        srv->in_use -= j->footprint;
        j->t_end = t;
        j->state = j->cancel.load() ? CM_JOB_CANCELLED : CM_JOB_DONE;
        j->error = j->state == CM_JOB_CANCELLED ? CM_ECANCELED : 0;
      }
      if (rc) {  // the batch failed: every job in it fails with the error
        std::vector<JobRecord*> all = b->active;
        for (JobRecord* j : admitted)
          if (std::find(all.begin(), all.end(), j) == all.end()) all.push_back(j);
        for (JobRecord* j : all) {
          srv->in_use -= j->footprint;
          j->t_end = t;
          j->state = CM_JOB_FAILED;
          j->error = rc;
          j->message = msg;
        }
        b->active.clear();
      }
    }
    if (!finished.empty() || rc) {
      srv->cv_done.notify_all();
      srv->cv_work.notify_all();
    }
    if (b->active.empty()) {
      batch_reset(*b);
      b->restarts = 0;
    }
  }
}

}  // namespace cm

extern "C" {

int cm_server_create(int device, int slots, double budget_gb, cm_server** out) {
  if (!out || slots < 1 || slots > 4096 || !(budget_gb > 0)) return fail(CM_EINVAL, "bad server arguments");
  int n = 0;
  CM_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(CM_EINVAL, "no such CUDA device");
  std::unique_ptr<cm_server> srv(new cm_server());
  srv->device = device;
  srv->max_active = slots;
  srv->budget = (size_t)(budget_gb * 1e9);
  *out = srv.release();
  return 0;
}

int cm_server_tune(cm_server* srv, int precision, const cm_tuning* t) {
  if (!srv || !t) return fail(CM_EINVAL, "null argument");
  if (precision != CM_PREC_FP64 && precision != CM_PREC_FP32) return fail(CM_EINVAL, "bad precision");
  if (t->wave < 0 || (t->wave > 0 && (t->wave < 1024 || t->wave > (1 << 24)))) return fail(CM_EINVAL, "wave out of range");
  if (t->tail_below < 0) return fail(CM_EINVAL, "tail_below < 0");
  if (t->tail_steps < 0 || t->tail_steps > 4096) return fail(CM_EINVAL, "tail_steps out of range");
  if (t->blocks_per_sm < 0 || t->blocks_per_sm > 32) return fail(CM_EINVAL, "blocks_per_sm out of range");
  if (t->pool < 0 || t->pool > 64) return fail(CM_EINVAL, "pool out of range");
  std::lock_guard<std::mutex> lk(srv->mu);
  srv->tune[precision] = *t;
  return 0;
}

int cm_server_destroy(cm_server* srv) {
  if (!srv) return 0;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    for (auto& kv : srv->jobs) kv.second->cancel.store(1);
    srv->stop = true;
  }
  srv->cv_work.notify_all();
  for (auto& kv : srv->batchers)
    if (kv.second->thread.joinable()) kv.second->thread.join();
  cudaSetDevice(srv->device);
  for (auto& kv : srv->batchers) {
    kv.second->release();
    cm_context_destroy(kv.second->ctx);
  }
  delete srv;
  return 0;
}

int cm_job_submit(cm_server* srv, const cm_context* scene, const cm_run_desc* d, int* out_job) {
  if (!srv || !scene || !d || !out_job) return fail(CM_EINVAL, "null argument");
  if (d->precision != CM_PREC_FP64 && d->precision != CM_PREC_FP32) return fail(CM_EINVAL, "bad precision");
  if (d->npix < 1) return fail(CM_EINVAL, "npix < 1");
  if (d->chamber < 0 || d->chamber >= (int)scene->regions.size() || scene->regions[d->chamber].parent != -1)
    return fail(CM_EINVAL, "bad chamber handle");
  if (d->hist_stride < 3 || d->hist_stride > 1026) return fail(CM_EINVAL, "hist_stride out of range");
  if (!d->pixel_center || !d->pixel_energy || !d->pixel_nprim || !d->pixel_nbins) return fail(CM_EINVAL, "null array");
  if (!(d->beam_width >= 0)) return fail(CM_EINVAL, "negative beam width");
  if (d->elevation || d->azimuth || d->escape_log)
    return fail(CM_EINVAL, "jobs tally the energy histograms only (no angle histograms or escape log)");
  if (d->pixel_first) return fail(CM_EINVAL, "jobs start every pixel at its primary 0 (no pixel_first)");
  std::unique_ptr<JobRecord> j(new JobRecord());
  j->options = scene->options;
  j->mott = scene->mott;
  j->tables = scene->tables;
  j->mats = scene->mats;
  j->msms = scene->msms;
  j->shapes = scene->shapes;
  j->regions = scene->regions;
  j->desc = *d;
  const int n = d->npix;
  j->center.assign(d->pixel_center, d->pixel_center + 3 * (size_t)n);
  j->energy.assign(d->pixel_energy, d->pixel_energy + n);
  j->nprim.assign(d->pixel_nprim, d->pixel_nprim + n);
  j->nbins.assign(d->pixel_nbins, d->pixel_nbins + n);
  if (d->pixel_key) j->keys.assign(d->pixel_key, d->pixel_key + n);
  {  // a job with bad pixels is refused at submission, not in the batch
    PixelPrep p;
    const int rc = prep_pixels(d, j->center.data(), j->energy.data(), j->nprim.data(), j->nbins.data(), d->hist_stride, p);
    if (rc) return rc;
  }
  j->desc.pixel_center = nullptr;
  j->desc.pixel_energy = nullptr;
  j->desc.pixel_nprim = nullptr;
  j->desc.pixel_nbins = nullptr;
  j->desc.pixel_key = d->pixel_key ? j->keys.data() : nullptr;
  j->desc.profile = 0;
  j->footprint = job_footprint(*d);
  memset(&j->stats, 0, sizeof(j->stats));
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stop) return fail(CM_ESTATE, "server is stopping");
    const std::pair<int, int> key(d->precision, scene->options);
    if (!srv->batchers.count(key)) {  // the first job of a precision and options starts its batcher
      std::unique_ptr<Batcher> b(new Batcher());
      b->precision = d->precision;
      b->options = scene->options;
      const int rc = cm_context_create(srv->device, &b->ctx);
      if (rc) return rc;
      b->ctx->options = scene->options;
      Batcher* bp = b.get();
      srv->batchers[key] = std::move(b);
      bp->thread = d->precision == CM_PREC_FP64 ? std::thread(batcher_worker<double>, srv, bp)
                                                 : std::thread(batcher_worker<float>, srv, bp);
    }
    j->id = srv->next_id++;
    j->t_submit = srv->now();
    *out_job = j->id;
    srv->queue.push_back(j->id);
    srv->jobs[j->id] = std::move(j);
  }
  srv->cv_work.notify_all();
  return 0;
}

int cm_job_poll(cm_server* srv, int job, cm_job_info* info) {
  if (!srv || !info) return fail(CM_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->jobs.find(job);
  if (it == srv->jobs.end()) return fail(CM_EINVAL, "no such job");
  fill_info(*it->second, info);
  return 0;
}

int cm_job_wait(cm_server* srv, int job, double timeout_s, cm_job_info* info) {
  if (!srv || !info) return fail(CM_EINVAL, "null argument");
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->jobs.find(job);
  if (it == srv->jobs.end()) return fail(CM_EINVAL, "no such job");
  JobRecord* j = it->second.get();
  auto finished = [&] { return j->state >= CM_JOB_DONE; };
  if (timeout_s < 0) srv->cv_done.wait(lk, finished);
  else srv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), finished);
  fill_info(*j, info);
  return 0;
}

int cm_job_cancel(cm_server* srv, int job) {
  if (!srv) return fail(CM_EINVAL, "null server");
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->jobs.find(job);
    if (it == srv->jobs.end()) return fail(CM_EINVAL, "no such job");
    JobRecord* j = it->second.get();
    if (j->state == CM_JOB_QUEUED) {
      for (auto q = srv->queue.begin(); q != srv->queue.end(); ++q)
        if (*q == job) {
          srv->queue.erase(q);
          break;
        }
      j->state = CM_JOB_CANCELLED;
      j->error = CM_ECANCELED;
      j->t_end = srv->now();
    } else if (j->state == CM_JOB_RUNNING) {
      j->cancel.store(1);  // its batcher stops its unstarted primaries after the current round
    }
  }
  srv->cv_done.notify_all();
  srv->cv_work.notify_all();
  return 0;
}

int cm_job_result(cm_server* srv, int job, uint32_t* back, uint32_t* fwd, cm_run_stats* stats) {
  if (!srv) return fail(CM_EINVAL, "null server");
  std::unique_ptr<JobRecord> j;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->jobs.find(job);
    if (it == srv->jobs.end()) return fail(CM_EINVAL, "no such job");
    if (it->second->state < CM_JOB_DONE) return fail(CM_ESTATE, "job still queued or running");
    j = std::move(it->second);
    srv->jobs.erase(it);
  }
  if (j->state != CM_JOB_DONE)
    return fail(j->error ? j->error : CM_ECANCELED, j->message.empty() ? "job did not complete" : j->message);
  if (back) memcpy(back, j->back.data(), j->back.size() * 4);
  if (fwd) memcpy(fwd, j->fwd.data(), j->fwd.size() * 4);
  if (stats) *stats = j->stats;
  return 0;
}

}  // extern "C"
