// cm_server.cuh -- job server for streams of scan jobs (included by cm_engine.cu).
//
// A server owns `slots` engine contexts on one GPU, each with its own stream,
// scene, electron waves and per-pixel buffers, all kept resident between jobs.
// Jobs (a scene plus a run description with host arrays) are admitted first in,
// first out as soon as a slot is free and the device memory the job needs fits
// the server's budget; the slots run their jobs concurrently, so the kernels of
// jobs that arrive while others are on the GPU overlap with them.  A job's
// tallies depend only on its scene, its pixels and their stream keys, so a job
// gives the same result alone and in any mix.
//
// Each slot is driven by one host thread: a run launches its context's cached
// loop graph on the slot's stream once and waits for it; cancelling a running
// job sets a flag in mapped host memory that the loop reads every iteration.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

namespace cm {

struct JobRecord {
  int id = -1;
  int state = CM_JOB_QUEUED;
  int error = 0;
  std::string message;
  // the scene, copied from the submitter's context
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
  int* running_cancel = nullptr;  // while the job runs: its slot context's mapped cancel flag (the device loop reads it)
};

// ask a job to stop: the host flag, and for a running job the flag its device loop reads (server lock held)
static void request_cancel(JobRecord* j) {
  j->cancel.store(1);
  if (j->running_cancel) *(volatile int*)j->running_cancel = 1;
}

// device buffers of one slot, grown to the largest job it has run
struct SlotBuffers {
  int npix = 0;
  size_t hist = 0;  // u32 per tally array
  double *center = nullptr, *e0 = nullptr, *e0ref = nullptr;
  unsigned long long *prefix = nullptr, *key = nullptr;
  int* nbins = nullptr;
  uint32_t *back = nullptr, *fwd = nullptr;
  void release() {
    cudaFree(center);
    cudaFree(e0);
    cudaFree(e0ref);
    cudaFree(prefix);
    cudaFree(key);
    cudaFree(nbins);
    cudaFree(back);
    cudaFree(fwd);
    *this = SlotBuffers();
  }
  int ensure(int n, size_t h) {
    if (n > npix) {
      cudaFree(center);
      cudaFree(e0);
      cudaFree(e0ref);
      cudaFree(prefix);
      cudaFree(key);
      cudaFree(nbins);
      center = e0 = e0ref = nullptr;
      prefix = key = nullptr;
      nbins = nullptr;
      CM_CUDA(cudaMalloc(&center, (size_t)n * 3 * 8));
      CM_CUDA(cudaMalloc(&e0, (size_t)n * 8));
      CM_CUDA(cudaMalloc(&e0ref, (size_t)n * 8));
      CM_CUDA(cudaMalloc(&prefix, ((size_t)n + 1) * 8));
      CM_CUDA(cudaMalloc(&key, (size_t)n * 8));
      CM_CUDA(cudaMalloc(&nbins, (size_t)n * 4));
      npix = n;
    }
    if (h > hist) {
      cudaFree(back);
      cudaFree(fwd);
      back = fwd = nullptr;
      CM_CUDA(cudaMalloc(&back, h * 4));
      CM_CUDA(cudaMalloc(&fwd, h * 4));
      hist = h;
    }
    return 0;
  }
};

}  // namespace cm

struct cm_server {
  int device = 0;
  size_t budget = 0;  // bytes the running jobs' own buffers may take
  size_t in_use = 0;
  std::vector<cm_context*> slot_ctx;
  std::vector<cm::SlotBuffers> slot_buf;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<int> queue;  // admission order
  std::map<int, std::unique_ptr<cm::JobRecord>> jobs;
  int next_id = 0;
  bool stop = false;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace cm {

// device bytes a job needs beyond its slot's resident waves: pixel arrays and tallies
static size_t job_footprint(const cm_run_desc& d) {
  return (size_t)d.npix * (3 * 8 + 8 + 8 + 8 + 8 + 4) + 2 * (size_t)d.npix * d.hist_stride * 4 + 4096;
}

template <typename R>
static int slot_run(cm_context* ctx, SlotBuffers& b, JobRecord& job) {
  const cm_run_desc& d = job.desc;
  PixelPrep p;
  int rc = prep_pixels(&d, job.center.data(), job.energy.data(), job.nprim.data(), job.nbins.data(), d.hist_stride, p);
  if (rc) return rc;
  const size_t h = (size_t)d.npix * d.hist_stride;
  if ((rc = b.ensure(d.npix, h))) return rc;
  cudaStream_t s = ctx->stream;
  CM_CUDA(cudaMemcpyAsync(b.center, p.center_nm.data(), p.center_nm.size() * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.e0, p.e0.data(), p.e0.size() * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.e0ref, p.e0ref.data(), p.e0ref.size() * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.prefix, p.prefix.data(), p.prefix.size() * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.key, p.key.data(), p.key.size() * 8, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemcpyAsync(b.nbins, job.nbins.data(), job.nbins.size() * 4, cudaMemcpyHostToDevice, s));
  CM_CUDA(cudaMemsetAsync(b.back, 0, h * 4, s));
  CM_CUDA(cudaMemsetAsync(b.fwd, 0, h * 4, s));
  cm_run_desc dd = d;
  dd.pixel_center = b.center;
  dd.pixel_energy = b.e0;
  dd.pixel_nbins = b.nbins;
  rc = run_device<R>(ctx, &dd, b.back, b.fwd, &job.stats, s, b.prefix, b.e0ref, b.key, p.total);
  if (rc) return rc;
  job.back.resize(h);
  job.fwd.resize(h);
  CM_CUDA(cudaMemcpyAsync(job.back.data(), b.back, h * 4, cudaMemcpyDeviceToHost, s));
  CM_CUDA(cudaMemcpyAsync(job.fwd.data(), b.fwd, h * 4, cudaMemcpyDeviceToHost, s));
  CM_CUDA(cudaStreamSynchronize(s));
  return 0;
}

static void slot_worker(cm_server* srv, int slot) {
  cudaSetDevice(srv->device);
  cm_context* ctx = srv->slot_ctx[slot];
  for (;;) {
    JobRecord* job = nullptr;
    {
      std::unique_lock<std::mutex> lk(srv->mu);
      // first in, first out: the head job starts when its buffers fit the budget
      srv->cv_work.wait(lk, [&] {
        if (srv->stop) return true;
        if (srv->queue.empty()) return false;
        const JobRecord& head = *srv->jobs[srv->queue.front()];
        return srv->in_use == 0 || srv->in_use + head.footprint <= srv->budget;
      });
      if (srv->stop) return;
      job = srv->jobs[srv->queue.front()].get();
      srv->queue.pop_front();
      srv->in_use += job->footprint;
      job->state = CM_JOB_RUNNING;
      job->t_start = srv->now();
      *(volatile int*)ctx->cancel_host = job->cancel.load();
      job->running_cancel = ctx->cancel_host;
    }
    srv->cv_work.notify_all();
    // the slot takes the job's scene; the device copy is rebuilt on the first run
    ctx->options = job->options;
    ctx->mott = job->mott;
    ctx->tables = job->tables;
    ctx->mats = job->mats;
    ctx->msms = job->msms;
    ctx->shapes = job->shapes;
    ctx->regions = job->regions;
    ctx->dirty();
    ctx->cancel = &job->cancel;
    const int rc = job->desc.precision == CM_PREC_FP64 ? slot_run<double>(ctx, srv->slot_buf[slot], *job)
                                                       : slot_run<float>(ctx, srv->slot_buf[slot], *job);
    ctx->cancel = nullptr;
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      job->running_cancel = nullptr;
      srv->in_use -= job->footprint;
      job->t_end = srv->now();
      job->error = rc;
      if (rc) job->message = cm_last_error();
      job->state = rc == 0 ? CM_JOB_DONE : rc == CM_ECANCELED ? CM_JOB_CANCELLED : CM_JOB_FAILED;
    }
    srv->cv_done.notify_all();
    srv->cv_work.notify_all();
  }
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

}  // namespace cm

extern "C" {

int cm_server_create(int device, int slots, double budget_gb, cm_server** out) {
  if (!out || slots < 1 || slots > 64 || !(budget_gb > 0)) return fail(CM_EINVAL, "bad server arguments");
  std::unique_ptr<cm_server> srv(new cm_server());
  srv->device = device;
  srv->budget = (size_t)(budget_gb * 1e9);
  for (int k = 0; k < slots; ++k) {
    cm_context* c = nullptr;
    const int rc = cm_context_create(device, &c);
    if (rc) {
      for (cm_context* x : srv->slot_ctx) cm_context_destroy(x);
      return rc;
    }
    srv->slot_ctx.push_back(c);
  }
  srv->slot_buf.resize(slots);
  cm_server* p = srv.release();
  for (int k = 0; k < slots; ++k) p->workers.emplace_back(slot_worker, p, k);
  *out = p;
  return 0;
}

int cm_server_destroy(cm_server* srv) {
  if (!srv) return 0;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    for (auto& kv : srv->jobs) request_cancel(kv.second.get());  // running jobs stop at their next iteration
    srv->stop = true;
  }
  srv->cv_work.notify_all();
  for (auto& t : srv->workers) t.join();
  cudaSetDevice(srv->device);
  for (auto& b : srv->slot_buf) b.release();
  for (cm_context* c : srv->slot_ctx) cm_context_destroy(c);
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
  if (d->elevation || d->azimuth || d->escape_log)
    return fail(CM_EINVAL, "jobs tally the energy histograms only (no angle histograms or escape log)");
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
  j->desc.pixel_center = nullptr;  // the worker points the run at the copies
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
      request_cancel(j);
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
  if (j->state != CM_JOB_DONE) return fail(j->error ? j->error : CM_ECANCELED, j->message.empty() ? "job did not complete" : j->message);
  if (back) memcpy(back, j->back.data(), j->back.size() * 4);
  if (fwd) memcpy(fwd, j->fwd.data(), j->fwd.size() * 4);
  if (stats) *stats = j->stats;
  return 0;
}

}  // extern "C"
