// cm_wave.cuh -- the wavefront: electron records, queues and the per-electron
// work of each event kernel.
//
// Every function here handles one electron and is host-callable; the kernels
// in cm_engine.cu are grid-stride loops over them with a DeviceSink that does
// warp-aggregated appends.  Reference paths relative to
// CudaMONSEL/CudaMONSEL/gov/nist/.
#pragma once
#include "cm_physics.cuh"

namespace cm {

// structure-of-arrays electron records (one per wave slot)
template <typename R>
struct Wave {
  double *px, *py, *pz;
  R *dx, *dy, *dz;
  R *E, *Ep;
  int *region, *pixel, *aux;
  uint32_t* step;
  unsigned long long* key;
  R *hx, *hy, *hz;
};

struct Counters {
  int n[2];              // electrons in each wave
  int nc[2][kSegments];  // of which in each segment (segment k holds slots [k W, k W + nc))
  int ns[kSegments];     // electrons the refill appends after the survivors of each segment
  int pool;
  int q[3];
  int error;
  int done;
  unsigned long long next_primary, total_primaries;
  unsigned long long steps, scatters, barriers, escapes, secondaries;
  unsigned long long iterations;
  unsigned long long units[4];
  unsigned long long step_units;  // electrons the several-steps kernel started with
  unsigned long long logged;      // escapes offered to the escape log
  unsigned long long slots, tail_slots;  // iteration slots the device-driven loop ran (all, tail)
  unsigned long long ended_zero, ended_limit;  // electrons ended by the zero-energy cut, by the step limit
  int fill;  // the refill fills the wave up to this many electrons (0: W); set by the job server's tail rounds
};

template <typename R>
struct El {
  double p[3];
  R d[3];
  R E, Ep;
  int region, pixel, aux;
  uint32_t step;
  unsigned long long key;
  R h[3];
};

template <typename R> CM_D El<R> load(const Wave<R>& w, int i) {
  El<R> e;
  e.p[0] = w.px[i]; e.p[1] = w.py[i]; e.p[2] = w.pz[i];
  e.d[0] = w.dx[i]; e.d[1] = w.dy[i]; e.d[2] = w.dz[i];
  e.E = w.E[i]; e.Ep = w.Ep[i];
  e.region = w.region[i]; e.pixel = w.pixel[i]; e.aux = w.aux[i];
  e.step = w.step[i]; e.key = w.key[i];
  e.h[0] = w.hx[i]; e.h[1] = w.hy[i]; e.h[2] = w.hz[i];
  return e;
}

// The fields a step starts from (position, direction, energy, region, pixel, step count, key).  Ep, aux
// and the hit normal are written by the flight for its event and read only by that event, so records
// moved between waves and the pool carry the live fields alone (60 of 80 bytes in FP32).
template <typename R> CM_D El<R> load_live(const Wave<R>& w, int i) {
  El<R> e;
  e.p[0] = w.px[i]; e.p[1] = w.py[i]; e.p[2] = w.pz[i];
  e.d[0] = w.dx[i]; e.d[1] = w.dy[i]; e.d[2] = w.dz[i];
  e.E = w.E[i];
  e.region = w.region[i]; e.pixel = w.pixel[i];
  e.step = w.step[i]; e.key = w.key[i];
  return e;
}

template <typename R> CM_D void store_live(const Wave<R>& w, int i, const El<R>& e) {
  w.px[i] = e.p[0]; w.py[i] = e.p[1]; w.pz[i] = e.p[2];
  w.dx[i] = e.d[0]; w.dy[i] = e.d[1]; w.dz[i] = e.d[2];
  w.E[i] = e.E;
  w.region[i] = e.region; w.pixel[i] = e.pixel;
  w.step[i] = e.step; w.key[i] = e.key;
}

// what an elastic or inelastic event reads: the live fields, the step's starting energy and the mechanism
template <typename R> CM_D El<R> load_event(const Wave<R>& w, int i) {
  El<R> e = load_live(w, i);
  e.Ep = w.Ep[i];
  e.aux = w.aux[i];
  return e;
}

enum { Q_EL = 0, Q_TAB = 1, Q_MISC = 2 };
enum { AUX_MECH = 1, AUX_BARRIER = 2, AUX_PASS = 3 };
CM_HD int aux_pack(int kind, int v) { return (kind << 24) | (v & 0xffffff); }
CM_HD int aux_kind(int a) { return a >> 24; }
CM_HD int aux_val(int a) { return a & 0xffffff; }

#ifdef CM_TRACE
// step records of a debugging build (never compiled into the library)
struct TraceRec {
  unsigned long long key;
  unsigned int step;
  int region, next, kind;
  double E, p[3], d[3];
};
#endif

// What changes from run to run: the pixels, the tallies and the loop's limits.  It sits in device memory
// (written before each run) and the kernels read it through RunView::io, so the launch graph of a run
// does not depend on it and an instantiated graph serves every run of the same scene and buffers.
struct RunIO {
  const double* pc;      // pixel centres, nm
  const double* pe0;     // beam energy, eV
  const double* pe0ref;  // histogram top edge in eV as the reference computes it
  const int* pnbins;
  const unsigned long long* prefix;
  const unsigned long long* pkey;  // per-pixel stream key
  const unsigned long long* pfirst;  // per-pixel index of its first primary (a scan resumed), or null: 0
  int npix;
  double width;          // nm
  uint32_t *back, *fwd;
  int stride;
  uint32_t *elev, *azim;       // per-pixel angle histograms (182 and 362 counts), or null
  cm_escape_record* log;       // escape log, or null
  long long logCap;
  // the device-driven loop (k_loop): iteration slots allowed, the tail threshold, queue kernels only to
  // the end, and a flag in host memory that cancels the run (null: not cancellable)
  long long max_slots;
  int tail_below;
  int queue_only;
  const volatile int* cancel;
  // A run of several jobs (the job server's shared wave; all null otherwise): per pixel its chamber, the
  // offset of its tally row (u32 elements into back/fwd) and its job; per job the electrons alive (a
  // primary or secondary counts from its start to its end), their steps (added when each ends) and a stop
  // flag that keeps its unstarted primaries out of the wave.
  const int* pchamber;
  const double* pwidth;  // Gaussian beam width per pixel, nm
  const unsigned long long* ptally;
  const int* pjob;
  unsigned long long* job_alive;
  unsigned long long* job_steps;
  const int* job_stop;
};

template <typename R>
struct RunView {
#ifdef CM_TRACE
  TraceRec* trace;
  int* ntrace;
  int tracecap;
#endif
  SceneView<R> s;
  Wave<R> w[2];
  Wave<R> pool;
  int* q[3];
  Counters* c;
  int W, poolCap;
  const RunIO* io;
};

// per-thread event counts, reduced once per warp by the kernels
struct StepCounts {
  unsigned long long steps = 0, scat = 0, bar = 0, esc = 0, sec = 0, zero = 0, limit = 0;
};

// Histogram::bin (Utility/Histogram.cu:73-80) over bins min + i*delta with
// Algorithm::binarySearch (Amphibian/Algorithm.cu:5-14): exact match or the
// insertion point.
CM_D int hist_bin(double max, int nbins, double val) {
  const double delta = max / nbins;
  int l = 0, r = nbins;
  while (l <= r) {
    const int mid = l + (r - l) / 2;
    const double bm = mid == 0 ? 0.0 : 0.0 + mid * delta;
    if (bm == val) return mid;
    if (bm < val) l = mid + 1;
    else r = mid - 1;
  }
  return l;
}

// BackscatterStats::actionPerformed for a BackscatterEvent (NISTMonte/BackscatterStats.cu:147-170):
// elevation and azimuth histograms, the log, then the forward or back energy histogram
template <typename R, typename Sink> CM_D void tally_escape(const RunView<R>& v, const El<R>& e, Sink& sink) {
  const RunIO& io = *v.io;
  const int px = e.pixel;
  const double E0ref = io.pe0ref[px];
  double val = (double)e.E;
  if (e.E == (R)io.pe0[px]) val = E0ref;  // electrons that never lost energy carry E0 exactly, as in the reference
  const double elevation = (kPi / 2) - atan2(e.p[2], sqrt((e.p[0] * e.p[0]) + (e.p[1] * e.p[1])));
  if (io.elev) {
    double azimuth = atan2(e.p[1], e.p[0]);
    if (azimuth < 0.0) azimuth = (2.0 * kPi) + azimuth;
    const int be = hist_bin(kPi, 180, elevation) + 1, ba = hist_bin(2.0 * kPi, 360, azimuth) + 1;
    if (be <= 181) sink.count(io.elev + (size_t)px * 182 + be);  // past the overflow slot: never counted
    if (ba <= 361) sink.count(io.azim + (size_t)px * 362 + ba);
  }
  if (io.log) {
    const unsigned long long k = sink.ticket(&v.c->logged);
    if (k < (unsigned long long)io.logCap) {
      cm_escape_record& r = io.log[k];
      r.electron = e.key;
      r.pixel = px;
      r.step = (int)e.step;
      r.energy_eV = val;
      for (int j = 0; j < 3; ++j) r.position[j] = e.p[j] * 1e-9;
      r.theta = atan2(sqrt((double)e.d[0] * (double)e.d[0] + (double)e.d[1] * (double)e.d[1]), (double)e.d[2]);
      r.phi = atan2((double)e.d[1], (double)e.d[0]);
    }
  }
  const int nb = io.pnbins[px];
  const int b = hist_bin(E0ref, nb, val) + 1;
  if (b > nb + 1) return;  // past the overflow slot: the reference writes out of bounds and never counts it
  uint32_t* h = elevation < (kPi / 2.0) ? io.fwd : io.back;
  sink.count(h + (io.ptally ? (size_t)io.ptally[px] : (size_t)px * io.stride) + b);
}

#ifdef CM_TRACE
template <typename R, typename Sink> CM_D void cm_trace(const RunView<R>& v, const El<R>& e, int next, int kind, Sink& sink) {
  const int k = sink.append(v.ntrace);
  if (k >= v.tracecap) return;
  TraceRec& t = v.trace[k];
  t.key = e.key; t.step = e.step; t.region = e.region; t.next = next; t.kind = kind; t.E = (double)e.E;
  for (int j = 0; j < 3; ++j) { t.p[j] = e.p[j]; t.d[j] = (double)e.d[j]; }
}
#endif

// job accounting of a run of several jobs: an electron of pixel px starts, or ends after `steps` steps
template <typename R, typename Sink> CM_D void job_start(const RunView<R>& v, int px, Sink& sink) {
  const RunIO& io = *v.io;
  if (io.job_alive) sink.add_by(io.job_alive, io.pjob[px], 1ull);
}
template <typename R, typename Sink> CM_D void job_end(const RunView<R>& v, int px, uint32_t steps, Sink& sink) {
  const RunIO& io = *v.io;
  if (!io.job_alive) return;
  const int j = io.pjob[px];
  sink.add_by(io.job_alive, j, ~0ull);  // minus one
  sink.add_by(io.job_steps, j, (unsigned long long)steps);
}

// the chamber a pixel's electrons fly in
template <typename R> CM_D int chamber_of(const RunView<R>& v, int px) {
  const RunIO& io = *v.io;
  return io.pchamber ? io.pchamber[px] : v.s.chamber;
}

// MONSEL_MaterialScatterModel::setCache (MONSEL_MaterialScatterModel.cu:44-62): the cumulative scatter rates
// of the model's mechanisms at E (1/nm) into cum[0..nmech); returns the total
template <typename R> CM_D R msm_cumulative_rates(const SceneView<R>& s, const Msm& m, R E, R* cum) {
  R total = 0;
  const R logE = mlog(E);
  for (int k = 0; k < m.nmech; ++k) {
    total += mech_rate(s, s.mechs[m.mech0 + k], E, logE);
    cum[k] = total;
  }
  return total;
}

// MONSEL_MaterialScatterModel::scatter (:93-134): the first mechanism whose cumulative rate reaches r
template <typename R> CM_D int mech_pick(const R* cum, int n, R r) {
  int idx = 0;
  while (idx < n - 1 && cum[idx] < r) ++idx;
  return idx;
}

// ---------------------------------------------------------------- flight
// MonteCarloSS::takeStep (NISTMonte/MonteCarloSS.cu:107-163) up to the event:
// region check, MONSEL_MaterialScatterModel::randomMeanPathLength, the
// candidate point, RegionBase::findEndOfStep, the slowing-down loss, the
// tracking cut; the step's end is queued for its event kernel, escapes are tallied.
// One step's flight on a record held in registers (p, d, E, step, region and key valid; the pixel too,
// or, when pixel_src is given, read from there if the electron escapes): the event queue of its end, or
// -1 when the electron ended here (escaped and tallied, stopped, trapped).
template <typename R, int D, typename Sink>
CM_D int flight_apply(const RunView<R>& v, El<R>& e, Sink& sink, StepCounts& sc, const int* pixel_src = nullptr) {
  const SceneView<R>& s = v.s;
  int reg = e.region;
  if (reg < 0 || !shape_contains<R, D>(s, s.regions[reg].shape, e.p))
    reg = containing_subregion<R, D>(s, chamber_of(v, pixel_src ? *pixel_src : e.pixel), e.p);
  if (reg < 0) return -1;
  const Msm& m = s.msms[s.regions[reg].msm];
  bool complete = false;
  double fp = 2.0 * kChamberRadiusNm;
  R total = 0;
  int idx = 0, kind = 0;
  {
    Rng<R> g(e.key, e.step, 0);
    R cum[kMaxMech];
    total = msm_cumulative_rates(s, m, e.E, cum);
    if (total != R(0)) {
      const R f = -mlog(g.next()) / total;
      if ((double)f < fp) fp = (double)f;
      // MONSEL_MaterialScatterModel::scatter (:93-134) picks the mechanism from the rates at the
      // step's starting energy with the stream's next deviate; it is drawn here, before the
      // geometry, so that the rates need not stay live (nothing else draws from this stream)
      idx = mech_pick(cum, m.nmech, g.next() * total);
      kind = s.mechs[m.mech0 + idx].kind;
    } else if (e.step > 1000000u) {  // MONSEL_MaterialScatterModel::randomMeanPathLength (:86-90)
      complete = true;
      ++sc.limit;
    } else if (!(e.E > R(0)) && e.step > 4096u) {
      // With no energy and no mechanism an electron only flies straight and is reflected by every
      // barrier it meets (ExpQMBarrierSM: perpE = 0 never transmits); trapped between two walls it
      // bounces until the 1e6-step limit above, one wave iteration per bounce.  It is ended here
      // once it has taken 4096 steps (one that would have reached the chamber later, tallied at
      // 0 eV, is lost; that needs more than 4096 steps and never occurred in the tests).  Counted in
      // cm_run_stats.ended_zero_energy.
      complete = true;
      ++sc.zero;
    }
  }
  double p1[3] = {e.p[0] + fp * (double)e.d[0], e.p[1] + fp * (double)e.d[1], e.p[2] + fp * (double)e.d[2]};
  double hn[3];
  bool clipped = false;
  const int next = find_end_of_step<R, D>(s, reg, e.p, p1, hn, &clipped);
  const double dd = sqrt((p1[0] - e.p[0]) * (p1[0] - e.p[0]) + (p1[1] - e.p[1]) * (p1[1] - e.p[1]) +
                         (p1[2] - e.p[2]) * (p1[2] - e.p[2]));
  const R dE = m.csd ? jln_compute(m.jln, (R)dd, e.E) : R(0);
  e.p[0] = p1[0]; e.p[1] = p1[1]; e.p[2] = p1[2];
  e.Ep = e.E;
  e.E += dE;
  e.step += 1;
  e.region = reg;
  ++sc.steps;
  if ((e.E < (R)m.minE) || complete) return -1;
  int queue;
  if (next == reg) {
    ++sc.scat;
    if (total == R(0)) {
      // A step without mechanisms (vacuum) that stopped at a boundary leading back into the
      // same region: the segment grazed a shape within less than SMALL_DISP, or starts on the
      // far face of one.  The reference repeats such zero-length steps until its 1e6-step
      // limit (MONSEL_MaterialScatterModel.cu:88); move past the boundary as takeStep does
      // after a crossing (MonteCarloSS.cu:145).
      if (clipped) {
        e.p[0] += kSmallDispNm * (double)e.d[0];
        e.p[1] += kSmallDispNm * (double)e.d[1];
        e.p[2] += kSmallDispNm * (double)e.d[2];
      }
      queue = Q_MISC;
      e.aux = aux_pack(AUX_PASS, 0);
    } else {
      if (kind == MECH_POLARON) return -1;  // GanachaudMokraniPolaronTrapSM::scatter: trapped, E = 0
      queue = kind == MECH_NISTMOTT ? Q_EL : kind == MECH_TABULATED ? Q_TAB : Q_MISC;
      e.aux = aux_pack(AUX_MECH, idx);
    }
  } else if (next >= 0) {
    ++sc.bar;
    queue = Q_MISC;
    e.aux = aux_pack(AUX_BARRIER, next);
    e.h[0] = (R)hn[0]; e.h[1] = (R)hn[1]; e.h[2] = (R)hn[2];
  } else {
    ++sc.esc;
    if (pixel_src) e.pixel = *pixel_src;
    tally_escape(v, e, sink);
#ifdef CM_TRACE
    cm_trace(v, e, next, 9, sink);
#endif
    return -1;
  }
#ifdef CM_TRACE
  cm_trace(v, e, next, queue * 100 + aux_kind(e.aux) * 10 + aux_val(e.aux) % 10, sink);
#endif
  return queue;
}

// The flight of wave slot i: reads what the step uses and writes back only what it changes
// (direction, pixel and key stay in place for the event kernels), then queues the event.
template <typename R, int D, typename Sink>
CM_D void flight_one(const RunView<R>& v, int cur, int i, Sink& sink, StepCounts& sc) {
  const Wave<R>& W = v.w[cur];
  El<R> e;
  e.p[0] = W.px[i]; e.p[1] = W.py[i]; e.p[2] = W.pz[i];
  e.d[0] = W.dx[i]; e.d[1] = W.dy[i]; e.d[2] = W.dz[i];
  e.E = W.E[i];
  e.step = W.step[i];
  e.region = W.region[i];
  e.key = W.key[i];
  const int queue = flight_apply<R, D>(v, e, sink, sc, W.pixel + i);  // the pixel is read only on escape
  if (queue < 0) {
    if (v.io->job_alive) job_end(v, W.pixel[i], e.step, sink);
    return;
  }
  W.px[i] = e.p[0]; W.py[i] = e.p[1]; W.pz[i] = e.p[2];
  W.E[i] = e.E; W.Ep[i] = e.Ep;
  W.region[i] = e.region; W.aux[i] = e.aux;
  W.step[i] = e.step;
  if (aux_kind(e.aux) == AUX_BARRIER) { W.hx[i] = e.h[0]; W.hy[i] = e.h[1]; W.hz[i] = e.h[2]; }
  const int slot = sink.append_q(v.c->q, queue);
  v.q[queue][slot] = i;
}

// wave segment of an electron in `region` at energy E: its material's class, split at kSegmentSplitEv
template <typename R> CM_D int wave_segment(const SceneView<R>& s, int region, R E) {
  const int cls = region >= 0 ? s.regions[region].cls : 0;
  return 2 * cls + (E < (R)kSegmentSplitEv ? 1 : 0);
}

// append a surviving electron to its segment of the next wave
template <typename R, typename Sink> CM_D void keep(const RunView<R>& v, int nxt, const El<R>& e, Sink& sink) {
  const int k = wave_segment(v.s, e.region, e.E);
  const int slot = sink.append_q(v.c->nc[nxt], k);
  store_live(v.w[nxt], k * v.W + slot, e);
}

// wave index of the i-th electron of a wave counted over its class segments in order
CM_D int wave_index(const Counters* c, int cur, int W, int i) {
  int k = 0;
  while (k < kSegments - 1 && i >= c->nc[cur][k]) {
    i -= c->nc[cur][k];
    ++k;
  }
  return k * W + i;
}

CM_D int survivors(const Counters* c, int nxt) {
  int n = 0;
  for (int k = 0; k < kSegments; ++k) n += c->nc[nxt][k];
  return n;
}

// push a secondary to the pool when MonteCarloSS::trackSecondaryElectron (:165-174) would track it
template <typename R, typename Sink>
CM_D void push_secondary(const RunView<R>& v, const El<R>& pe, const R sd[3], R sE, Sink& sink, StepCounts& sc) {
  const Msm& m = v.s.msms[v.s.regions[pe.region].msm];
  if (!(sE > (R)m.minE)) return;
  El<R> se;
  se.p[0] = pe.p[0]; se.p[1] = pe.p[1]; se.p[2] = pe.p[2];
  se.d[0] = sd[0]; se.d[1] = sd[1]; se.d[2] = sd[2];
  se.E = sE; se.Ep = sE;
  se.region = pe.region;
  se.pixel = pe.pixel;
  se.aux = 0;
  se.step = 0;
  se.key = mix64(pe.key ^ (0x9E3779B97F4A7C15ULL * (unsigned long long)pe.step));
  se.h[0] = se.h[1] = se.h[2] = 0;
  const int slot = sink.append(&v.c->pool);
  if (slot >= v.poolCap) {
    sink.error(&v.c->error, -5 /* CM_EOVERFLOW */);
    return;
  }
  store_live(v.pool, slot, se);
  job_start(v, pe.pixel, sink);
  ++sc.sec;
}

// The events of a step on a record in registers (after its flight: step already counted, so the
// event's stream is (key, step - 1, 1)).  Each returns whether the electron lives on.

// SelectableElasticSM events
template <typename R> CM_D bool elastic_apply(const RunView<R>& v, El<R>& e) {
  const SceneView<R>& s = v.s;
  const Msm& m = s.msms[s.regions[e.region].msm];
  const Mech& k = s.mechs[m.mech0 + aux_val(e.aux)];
  Rng<R> g(e.key, e.step - 1, 1);
  elastic_scatter(s, k, e.d, e.Ep, g);
  return !(e.E < (R)m.minE);
}

// TabulatedInelasticSM events
template <typename R, typename Sink> CM_D bool inelastic_apply(const RunView<R>& v, El<R>& e, Sink& sink, StepCounts& sc) {
  const SceneView<R>& s = v.s;
  const Msm& m = s.msms[s.regions[e.region].msm];
  const Mech& k = s.mechs[m.mech0 + aux_val(e.aux)];
  Rng<R> g(e.key, e.step - 1, 1);
  R sd[3], sE;
  const bool made = tabulated_scatter(s, k, e.d, e.E, sd, sE, g);
  if (made) push_secondary(v, e, sd, sE, sink, sc);
  return !(e.E < (R)m.minE);
}

// barrier crossings, FittedInelSM, phonon, and steps that end without a mechanism
template <typename R, int D, typename Sink> CM_D bool misc_apply(const RunView<R>& v, El<R>& e, Sink& sink, StepCounts& sc) {
  const SceneView<R>& s = v.s;
  const Msm& m = s.msms[s.regions[e.region].msm];
  const int kind = aux_kind(e.aux);
  Rng<R> g(e.key, e.step - 1, 1);
  if (kind == AUX_BARRIER) {
    // MonteCarloSS::takeStep (:143-156): barrierScatter, a nudge along the new direction, region update
    const double hn[3] = {(double)e.h[0], (double)e.h[1], (double)e.h[2]};
    e.region = barrier_scatter(s, m, e.p, e.d, e.E, e.region, aux_val(e.aux), hn, g);
    e.p[0] += kSmallDispNm * (double)e.d[0];
    e.p[1] += kSmallDispNm * (double)e.d[1];
    e.p[2] += kSmallDispNm * (double)e.d[2];
    if (!shape_contains<R, D>(s, s.regions[e.region].shape, e.p))
      e.region = containing_subregion<R, D>(s, chamber_of(v, e.pixel), e.p);
    return true;
  }
  if (kind == AUX_MECH) {
    const Mech& k = s.mechs[m.mech0 + aux_val(e.aux)];
    if (k.kind == MECH_FITTED) {  // FittedInelSM::scatter (FittedInelSM.cu:13-18)
      const R phi = R(2) * R(kPi) * g.next();
      const R theta = iso_angle(g.next());
      R sd[3];
      dir_from_angles(sd, theta, phi);
      push_secondary(v, e, sd, (R)(k.energySEgen + k.eFermi), sink, sc);
    } else if (k.kind == MECH_PHONON) {
      phonon_scatter(k, e.d, e.E, e.Ep, g);
    }
  }
  return !(e.E < (R)m.minE);
}

// the queue kernels' events: the record of queue entry j, its event, and the survivor kept
template <typename R, typename Sink> CM_D void elastic_one(const RunView<R>& v, int cur, int j, Sink& sink) {
  El<R> e = load_event(v.w[cur], v.q[Q_EL][j]);
  if (elastic_apply(v, e)) keep(v, cur ^ 1, e, sink);
  else job_end(v, e.pixel, e.step, sink);
}

template <typename R, typename Sink> CM_D void inelastic_one(const RunView<R>& v, int cur, int j, Sink& sink, StepCounts& sc) {
  El<R> e = load_event(v.w[cur], v.q[Q_TAB][j]);
  if (inelastic_apply(v, e, sink, sc)) keep(v, cur ^ 1, e, sink);
  else job_end(v, e.pixel, e.step, sink);
}

template <typename R, int D, typename Sink>
CM_D void misc_one(const RunView<R>& v, int cur, int j, Sink& sink, StepCounts& sc) {
  El<R> e = load(v.w[cur], v.q[Q_MISC][j]);
  if (misc_apply<R, D>(v, e, sink, sc)) keep(v, cur ^ 1, e, sink);
  else job_end(v, e.pixel, e.step, sink);
}

// Up to nsteps whole steps (flight and event) of wave slot i in one thread, the survivor kept.  The
// tail of a run, when too few electrons are left to fill the GPU, goes this way: the same steps
// with the same random streams as the queue kernels, without a launch and a queue per event.
template <typename R, int D, typename Sink>
CM_D void steps_one(const RunView<R>& v, int cur, int i, int nsteps, Sink& sink, StepCounts& sc) {
  El<R> e = load_live(v.w[cur], i);
  for (int k = 0; k < nsteps; ++k) {
    const int q = flight_apply<R, D>(v, e, sink, sc);
    const bool alive = q < 0 ? false
                             : q == Q_EL ? elastic_apply(v, e)
                                         : q == Q_TAB ? inelastic_apply(v, e, sink, sc) : misc_apply<R, D>(v, e, sink, sc);
    if (!alive) {
      job_end(v, e.pixel, e.step, sink);
      return;
    }
  }
  keep(v, cur ^ 1, e, sink);
}

// refill plan of the next wave: secondaries from the pool first; new primaries
// only once the pool is empty, and at most W/32 per iteration so that the
// cascades of one batch of primaries do not all peak together
CM_D void refill_plan(const Counters* c, int nxt, int W, int poolCap, int& nn, int& take_se, int& take_p) {
  nn = survivors(c, nxt);
  const int cap = c->fill > 0 && c->fill < W ? c->fill : W;
  const int room = cap - nn > 0 ? cap - nn : 0;
  const int pool = c->pool < poolCap ? c->pool : poolCap;  // an overflowed pool holds poolCap valid entries
  take_se = pool < room ? pool : room;
  const unsigned long long rem = c->total_primaries - c->next_primary;
  int left = pool > take_se ? 0 : room - take_se;
  const int ramp = W / 32 > 1 ? W / 32 : 1;
  if (left > ramp) left = ramp;
  take_p = rem < (unsigned long long)left ? (int)rem : left;
}

// the j-th electron the refill adds to the next wave: a secondary from the top
// of the pool or a new primary, appended after the survivors of its segment
template <typename R, int D, typename Sink>
CM_D void spawn_one(const RunView<R>& v, int nxt, int j, int take_se, int poolTop, unsigned long long first,
                    Sink& sink) {
  if (j < take_se) {
    const El<R> se = load_live(v.pool, poolTop - 1 - j);
    const int seg = wave_segment(v.s, se.region, se.E);
    store_live(v.w[nxt], seg * v.W + v.c->nc[nxt][seg] + sink.append_q(v.c->ns, seg), se);
    return;
  }
  // GaussianBeam::createElectron (NISTMonte/GaussianBeam.cu:52-65) + initializeTrajectory (MonteCarloSS.cu:99-105)
  const RunIO& io = *v.io;
  const unsigned long long gi = first + (unsigned long long)(j - take_se);
  int lo = 0, hi = io.npix;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (io.prefix[mid] <= gi) lo = mid;
    else hi = mid;
  }
  const int px = lo;
  if (io.job_stop && io.job_stop[io.pjob[px]]) return;  // a stopped job starts no more primaries
  const unsigned long long k = gi - io.prefix[px] + (io.pfirst ? io.pfirst[px] : 0ull);
  El<R> e;
  e.key = mix64(io.pkey[px] + mix64(k + 1));
  Rng<R> g(e.key, 0xFFFFFFFFu, 0);
  const double u1 = (double)g.next(), u2 = (double)g.next();
  const double r = sqrt(-2. * log(u1)) * (io.pwidth ? io.pwidth[px] : io.width);
  const double th = 2.0 * kPi * u2;
  e.p[0] = io.pc[3 * px] + r * cos(th);
  e.p[1] = io.pc[3 * px + 1] + r * sin(th);
  e.p[2] = io.pc[3 * px + 2];
  e.d[0] = 0; e.d[1] = 0; e.d[2] = 1;
  e.E = (R)io.pe0[px];
  e.Ep = e.E;
  e.region = containing_subregion<R, D>(v.s, chamber_of(v, px), e.p);
  e.pixel = px;
  e.aux = 0;
  e.step = 0;
  e.h[0] = e.h[1] = e.h[2] = 0;
  const int seg = wave_segment(v.s, e.region, e.E);
  store_live(v.w[nxt], seg * v.W + v.c->nc[nxt][seg] + sink.append_q(v.c->ns, seg), e);
  job_start(v, px, sink);
}

// end of an iteration: counters of the next wave, reset of this one (steps: the iteration ran k_steps)
CM_D void tail_update(Counters* c, int cur, int W, int poolCap, bool steps) {
  const int nxt = cur ^ 1;
  int nn, take_se, take_p;
  refill_plan(c, nxt, W, poolCap, nn, take_se, take_p);
  if (c->pool > poolCap) c->pool = poolCap;
  if (!c->done) {
    if (steps) c->step_units += (unsigned long long)c->n[cur];
    else c->units[0] += (unsigned long long)c->n[cur];
    c->units[1] += (unsigned long long)c->q[0];
    c->units[2] += (unsigned long long)c->q[1];
    c->units[3] += (unsigned long long)c->q[2];
    c->iterations += 1;
  }
  (void)nn;
  int appended = 0;  // survivors and refills as appended (a stopped job's primaries are not)
  for (int k = 0; k < kSegments; ++k) {
    c->nc[nxt][k] += c->ns[k];
    c->ns[k] = 0;
    c->nc[cur][k] = 0;
    appended += c->nc[nxt][k];
  }
  c->n[nxt] = appended;
  c->pool -= take_se;
  c->next_primary += (unsigned long long)take_p;
  c->n[cur] = 0;
  c->q[0] = c->q[1] = c->q[2] = 0;
  c->done = (c->n[nxt] == 0 && c->pool == 0 && c->next_primary == c->total_primaries) ? 1 : 0;
}

}  // namespace cm
