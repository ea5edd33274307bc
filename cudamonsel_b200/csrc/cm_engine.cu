// cm_engine.cu -- wavefront electron-transport engine for sm_100a and its C ABI.
//
// Replaces MonteCarloSS::runMultipleTrajectories (NISTMonte/MonteCarloSS.cu:
// 107-231) for a batch of beam landing points.  One "wave" of live electrons
// is kept as structure-of-arrays in HBM.  Each iteration runs
//
//   flight   : region check, scatter rates, free path, boundary search, CSD
//              loss, escape tally; classifies every electron's step end and
//              appends it (warp-aggregated) to one event queue
//   elastic  : SelectableElasticSM/NISTMottRS events
//   inelastic: TabulatedInelasticSM events (secondaries -> pool)
//   misc     : barrier crossings, FittedInelSM, phonon, pass-through
//   spawn    : refill the next wave from the secondary pool, then primaries
//   tail     : swap counters
//
// Survivors of every event kernel are appended compactly into the other wave
// buffer, so the next flight reads fully coalesced SoA.  Every electron draws
// from its own Philox stream (key = primary or parent lineage, counter =
// step), so results do not depend on scheduling or on what else is in the wave.
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <chrono>
#include <string>
#include <vector>

#include "../../include/cudamonsel_b200.h"
#include "cm_wave.cuh"

namespace cg = cooperative_groups;

namespace cm {

// ------------------------------------------------------------------ units
static const double kEV = 1.60217653e-19;          // PhysicalConstants::ElectronCharge
static const double kFromSIeV = 1.0 / 1.60217653e-19;  // FromSI::EV
// the small tables (prefix of the table blob) the event kernels stage into shared memory
static const size_t kStageBytes = 48 * 1024;
static const double kToSIkeV = 1.60217653e-19 * 1.0e3;
static const double kBohr = 5.291772083e-11;
static const double kAvogadro = 6.0221415e23;
static const double kBoltzmann = 1.3806505e-23;
static const double kElectronMass = 9.1093826e-31;
static const double kHbar = 1.05457266e-34;

static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CM_CUDA(call)                                                                            \
  do {                                                                                           \
    cudaError_t _e = (call);                                                                     \
    if (_e != cudaSuccess) return fail(CM_ECUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

// ------------------------------------------------------------------ host scene registry (SI)
struct HTable {
  int dim;
  int n[3];
  std::vector<double> x[3];
  std::vector<double> v;
  double domain[3][2];
  double range[2];
  int role;  // 0 none, 1 IIMFP, 2 reduced dE, 3 theta, 4 SE E0
};

struct HMaterial {
  std::vector<int> Z;
  std::vector<double> A, wf, core;
  double density, workfunction, ecb, bandgap;
};

struct HMech {
  int kind;
  int method;
  double energyOffset;
  int tables[4];
  double energySEgen, breakE;
  double ratemult, phononE, temperature, eps0, epsInf;
  double prefactor, extinction;
};

struct HMsm {
  int material;
  std::vector<HMech> mechs;
  int csd;
  double breakE;
  bool minSet;
  double minE;
  int classical;
  double lambda;
};

struct HShape {
  int kind;
  double c[3], r;
  std::vector<double> n, p;  // planes
  int a, b;
  double e0[3], ax[3], nax[3], radius;  // cylinder (SI); nax as NormalCylindricalShape computed it
  double len2;                          // |axis|^2 as the cylinder was built (rotations keep it)
};

struct HRegion {
  int parent, msm, shape;
  std::vector<int> children;
};

struct HMott {
  std::vector<double> spwem, x1;
};

template <typename R>
struct DevScene {
  std::vector<void*> allocs;
  SceneView<R> view;
  unsigned long long gen = 0;  // counts builds: a cached launch graph holds the view of one build
  bool valid = false;
  bool host = false;  // tables in host memory (only for host-side checks of the device code)
  void release() {
    for (void* p : allocs) host ? free(p) : (void)cudaFree(p);
    allocs.clear();
    valid = false;
  }
};

// what a cached launch graph was built for: a graph holds the RunView of these buffers and scene build
struct LoopKey {
  unsigned long long scene_gen;
  int chamber, grid, inel_grid, tail_steps, stage;
  bool operator==(const LoopKey& o) const {
    return scene_gen == o.scene_gen && chamber == o.chamber && grid == o.grid && inel_grid == o.inel_grid &&
           tail_steps == o.tail_steps && stage == o.stage;
  }
};

template <typename R>
struct RunBuffers {
  int cap = 0, poolCap = 0;
  std::vector<void*> allocs;
  Wave<R> w[2], pool;
  int* q[3] = {nullptr, nullptr, nullptr};
  RunIO* io = nullptr;  // device copy of the run's RunIO
  // the device-driven transport loop, instantiated once and launched by every run that matches its key
  cudaGraph_t loop_graph = nullptr;
  cudaGraphExec_t loop_exec = nullptr;
  LoopKey loop_key{};
  void drop_graph() {
    if (loop_exec) cudaGraphExecDestroy(loop_exec);
    if (loop_graph) cudaGraphDestroy(loop_graph);
    loop_exec = nullptr;
    loop_graph = nullptr;
  }
  void release() {
    drop_graph();
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
    io = nullptr;
    cap = poolCap = 0;
  }
};

}  // namespace cm

using namespace cm;

struct cm_context {
  int device = 0;
  int options = 0;
  int nsm = 148;
  std::map<int, HMott> mott;
  std::vector<HTable> tables;
  std::vector<HMaterial> mats;
  std::vector<HMsm> msms;
  std::vector<HShape> shapes;
  std::vector<HRegion> regions;
  DevScene<double> d64;
  DevScene<float> d32;
  RunBuffers<double> rb64;
  RunBuffers<float> rb32;
  Counters* counters = nullptr;
  Counters* counters_host = nullptr;
  RunIO* io_host = nullptr;        // pinned staging of the run's RunIO
  cudaStream_t stream = nullptr;
  cudaStream_t cap_stream = nullptr;  // stream the launch graphs are captured on
  const std::atomic<int>* cancel = nullptr;  // set by a job server for the running job
  int* cancel_host = nullptr;      // mapped host flag the device loop reads (the server sets it on cancel)
  const int* cancel_dev = nullptr; // its device address
  cm_tuning tune[2] = {{0, 0, 0, 0, 0.0}, {0, 0, 0, 0, 0.0}};  // launch settings per precision (0: default)
  // boxes of plane sets by their planes (normals then points): a job server's batch scene holds many
  // copies of the same shapes and is rebuilt as jobs join, and each box is a vertex enumeration
  std::map<std::vector<double>, std::array<double, 6>> box_memo;
  void dirty() {
    d64.release();
    d32.release();
  }
};

// ------------------------------------------------------------------ scene upload
namespace cm {

// An NVTX range over the scope: the phases of a run (scene upload, run buffers, launch graph, transport,
// tally copies), autotuner trials and job-server rounds appear by name on a timeline (Nsight Systems,
// ncu's NVTX filters); without a tool attached a range costs a call that returns at once.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

template <typename T>
static int dev_copy(std::vector<void*>& allocs, const std::vector<T>& v, const T** out, bool host = false) {
  void* p = nullptr;
  size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
  if (host) {
    p = malloc(bytes);
    allocs.push_back(p);
    if (!v.empty()) memcpy(p, v.data(), v.size() * sizeof(T));
    *out = (const T*)p;
    return 0;
  }
  CM_CUDA(cudaMalloc(&p, bytes));
  allocs.push_back(p);
  if (!v.empty()) CM_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  *out = (const T*)p;
  return 0;
}

// JoyLuoNieminenCSD::init (JMONSEL/JoyLuoNieminenCSD.cu:42-82) in SI, converted to eV/nm
static Jln make_jln(const HMaterial& mt, double breakE) {
  Jln c;
  memset(&c, 0, sizeof(c));
  c.nce = (int)mt.Z.size();
  double bh = -mt.ecb;
  c.minE = bh * kFromSIeV;
  if (c.nce == 0) return c;
  double bhplus1eV = bh + kEV * 1.;
  if (breakE < bhplus1eV) breakE = bhplus1eV;
  double gamma = 0.;
  for (int i = 0; i < c.nce; ++i) {
    double z = mt.Z[i];
    double J = mt.Z[i] < 13 ? kEV * (11.5 * z) : kEV * (9.76 * z + 58.8 * pow(z, -0.19));
    double recipJ = 1.166 / J;
    double beta = 1. - (recipJ * bhplus1eV);
    double coef = 2.01507E-28 * mt.density * mt.wf[i] * mt.Z[i] / mt.A[i];
    gamma += coef * log((recipJ * breakE) + beta);
    c.coef[i] = coef * 1e-9 / (kEV * kEV);
    c.recipJ[i] = recipJ * kEV;
    c.beta[i] = beta;
  }
  gamma /= pow(breakE, 3.5);
  c.gamma = gamma * 1e-9 * pow(kEV, 1.5);
  c.breakE = breakE * kFromSIeV;
  return c;
}

static double efermi(const HMaterial& m) { return -m.ecb - m.workfunction; }

// NISTMottRS constructor members (JMONSEL/NISTMottRS.cu:76-91) for methods 1..3, SI
static void mott_constants(int Z, const HMott& hm, Mott& m) {
  m.Z = Z;
  m.zp17 = pow(Z, 1.7);
  m.zp2 = pow(Z, 2.0);
  m.zp3 = pow(Z, 3.0);
  const double dl50 = log(0.050 * kToSIkeV);
  const double param = (log(20.0 * kToSIkeV) - dl50) / 60.0;
  for (int method = 0; method < 4; ++method) {
    // 50 eV for method 1, 100 eV for methods 2 and 3 (NISTMottRS.cu:82)
    const double ext = kEV * (method <= 1 ? 50. : 100.);
    // ULagrangeInterpolation::d1 at the extrapolation energy, in double on the host
    const double x = log(ext);
    const double reducedx = (x - dl50) / param;
    int index0 = (int)reducedx - 1;
    if (index0 < 0) index0 = 0;
    if (index0 > 61 - 4) index0 = 61 - 4;
    double xx = reducedx - index0;
    const double* f = hm.spwem.data() + index0;
    int ns = (int)round(xx);
    if (ns < 0) ns = 0;
    else if (ns > 3) ns = 3;
    double c[4] = {f[0], f[1], f[2], f[3]}, d[4] = {f[0], f[1], f[2], f[3]};
    double y = c[ns--], dy = 0;
    for (int mm = 1; mm <= 3; mm++) {
      for (int i = 0; i <= 3 - mm; i++) {
        double ho = i - xx, hp = i + mm - xx, w = c[i + 1] - d[i];
        d[i] = -hp * w / mm;
        c[i] = -ho * w / mm;
      }
      dy = (2 * ns < (3 - 1 - mm)) ? c[ns + 1] : d[ns--];
      y += dy;
    }
    const double mottXS = (kBohr * kBohr) * y;
    const double e = ext * (1.0 / (1.60217653e-19 * 1.0e3));
    const double re = sqrt(e);
    const double browning = 3.0e-22 * m.zp17 / (e + 0.005 * m.zp17 * re + 0.0007 * m.zp2 / re);
    m.sfBrowning[method] = mottXS / browning;
    m.mottXSatMin[method] = y;
    m.extrapolateBelowEnergy[method] = ext * kFromSIeV;
  }
  const double zz = Z;
  const double zp = pow(zz, 1.0 / 3.0);
  m.rutherfordA = 7.670843088080456e-38 * zp * (1.0 + zz) * kFromSIeV;
  m.rutherfordB = 5.44967975966321e-19 * zp * zp * kFromSIeV;
  m.rutherfordAlpha = 5.44968e-19 * pow(Z, 2.0 / 3.0) * kFromSIeV;
}

// ---- bounding boxes (SI), used only to skip shapes a step cannot reach
struct Box {
  double lo[3], hi[3];
};

static const double kBoxWorld = 1.0;  // m: steps never leave |x| < 0.3 m (0.1 m chamber + a 0.2 m step)

static Box box_world() { return Box{{-kBoxWorld, -kBoxWorld, -kBoxWorld}, {kBoxWorld, kBoxWorld, kBoxWorld}}; }

// vertices of {x : n_i . (x - p_i) <= 0} clipped to the world box, by intersecting plane triples
static Box planes_box(const HShape& s) {
  std::vector<std::array<double, 6>> pl;  // n, p
  for (size_t i = 0; i < s.n.size() / 3; ++i)
    pl.push_back({s.n[3 * i], s.n[3 * i + 1], s.n[3 * i + 2], s.p[3 * i], s.p[3 * i + 1], s.p[3 * i + 2]});
  for (int a = 0; a < 3; ++a)
    for (int sg = -1; sg <= 1; sg += 2) {
      std::array<double, 6> q = {0, 0, 0, 0, 0, 0};
      q[a] = sg;
      q[3 + a] = sg * kBoxWorld;
      pl.push_back(q);
    }
  Box b{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}};
  const size_t n = pl.size();
  for (size_t i = 0; i < n; ++i)
    for (size_t j = i + 1; j < n; ++j)
      for (size_t k = j + 1; k < n; ++k) {
        const double* A = pl[i].data();
        const double* B = pl[j].data();
        const double* C = pl[k].data();
        const double det = A[0] * (B[1] * C[2] - B[2] * C[1]) - A[1] * (B[0] * C[2] - B[2] * C[0]) +
                           A[2] * (B[0] * C[1] - B[1] * C[0]);
        if (fabs(det) < 1e-12) continue;
        const double da = A[0] * A[3] + A[1] * A[4] + A[2] * A[5];
        const double db = B[0] * B[3] + B[1] * B[4] + B[2] * B[5];
        const double dc = C[0] * C[3] + C[1] * C[4] + C[2] * C[5];
        double x[3];
        x[0] = (da * (B[1] * C[2] - B[2] * C[1]) - A[1] * (db * C[2] - B[2] * dc) + A[2] * (db * C[1] - B[1] * dc)) / det;
        x[1] = (A[0] * (db * C[2] - B[2] * dc) - da * (B[0] * C[2] - B[2] * C[0]) + A[2] * (B[0] * dc - db * C[0])) / det;
        x[2] = (A[0] * (B[1] * dc - db * C[1]) - A[1] * (B[0] * dc - db * C[0]) + da * (B[0] * C[1] - B[1] * C[0])) / det;
        bool in = true;
        for (size_t m = 0; m < n && in; ++m) {
          const double* P = pl[m].data();
          const double d = P[0] * (x[0] - P[3]) + P[1] * (x[1] - P[4]) + P[2] * (x[2] - P[5]);
          const double scale = 1e-9 * (1.0 + fabs(x[0]) + fabs(x[1]) + fabs(x[2]));
          in = d <= scale;
        }
        if (!in) continue;
        for (int a = 0; a < 3; ++a) {
          b.lo[a] = std::min(b.lo[a], x[a]);
          b.hi[a] = std::max(b.hi[a], x[a]);
        }
      }
  return b;  // empty (lo > hi) when the plane set holds nothing inside the world box
}

// planes_box, remembered by the context for plane sets it has boxed before
static Box planes_box_memo(cm_context* ctx, const HShape& s) {
  std::vector<double> key(s.n);
  key.insert(key.end(), s.p.begin(), s.p.end());
  auto it = ctx->box_memo.find(key);
  if (it != ctx->box_memo.end()) {
    const auto& v = it->second;
    return Box{{v[0], v[1], v[2]}, {v[3], v[4], v[5]}};
  }
  const Box b = planes_box(s);
  if (ctx->box_memo.size() > 200000) ctx->box_memo.clear();  // bounded over a long-lived server
  ctx->box_memo.emplace(std::move(key), std::array<double, 6>{b.lo[0], b.lo[1], b.lo[2], b.hi[0], b.hi[1], b.hi[2]});
  return b;
}

static Box shape_box(cm_context* ctx, int id) {
  const HShape& s = ctx->shapes[id];
  Box b;
  switch (s.kind) {
    case SHAPE_PLANES:
      return planes_box_memo(ctx, s);
    case SHAPE_SPHERE:
      for (int a = 0; a < 3; ++a) {
        b.lo[a] = s.c[a] - s.r;
        b.hi[a] = s.c[a] + s.r;
      }
      return b;
    case SHAPE_CYLINDER:  // both end discs lie in the spheres of radius r about the end points
      for (int a = 0; a < 3; ++a) {
        b.lo[a] = std::min(s.e0[a], s.e0[a] + s.ax[a]) - s.radius;
        b.hi[a] = std::max(s.e0[a], s.e0[a] + s.ax[a]) + s.radius;
      }
      return b;
    case SHAPE_INTERSECTION:
    case SHAPE_UNION: {
      if (s.kind == SHAPE_INTERSECTION) {
        // an intersection of plane sets is one convex polytope: box its vertices, which is far
        // tighter than intersecting the boxes of slanted half-spaces (a sidewall alone spans the world)
        HShape all;
        all.kind = SHAPE_PLANES;
        std::vector<int> todo{id};
        bool planar = true;
        while (!todo.empty() && planar) {
          const HShape& h = ctx->shapes[todo.back()];
          todo.pop_back();
          if (h.kind == SHAPE_INTERSECTION) {
            todo.push_back(h.a);
            todo.push_back(h.b);
          } else if (h.kind == SHAPE_PLANES) {
            all.n.insert(all.n.end(), h.n.begin(), h.n.end());
            all.p.insert(all.p.end(), h.p.begin(), h.p.end());
          } else {
            planar = false;
          }
        }
        if (planar) return planes_box_memo(ctx, all);
      }
      const Box x = shape_box(ctx, s.a), y = shape_box(ctx, s.b);
      for (int a = 0; a < 3; ++a) {
        b.lo[a] = s.kind == SHAPE_UNION ? std::min(x.lo[a], y.lo[a]) : std::max(x.lo[a], y.lo[a]);
        b.hi[a] = s.kind == SHAPE_UNION ? std::max(x.hi[a], y.hi[a]) : std::min(x.hi[a], y.hi[a]);
      }
      return b;
    }
  }
  return box_world();
}

template <typename R>
static int build_scene(cm_context* ctx, DevScene<R>& ds) {
  if (ds.valid) return 0;
  NvtxRange range("cm scene upload");
  ds.release();
  std::vector<R> blob;
  std::vector<double> dbl;  // SceneView::dbl
  // The blob holds every table's abscissae and values and the NIST Mott cross sections.  Pieces are
  // built apart and laid out small first: the prefix that fits kStageBytes is what the event kernels
  // copy into shared memory (the rest, such as a large 3-D angle table, is read through L1/L2).
  struct Piece {
    std::vector<R> data;
    std::vector<int*> offs;   // offsets to patch
    std::vector<int> rel;     // relative offsets of those fields in data
  };
  std::vector<Piece> pieces;
  // tables, converted by role to eV / nm units
  std::vector<Table> tabs(ctx->tables.size());
  for (size_t ti = 0; ti < ctx->tables.size(); ++ti) {
    const auto& t = ctx->tables[ti];
    Table& d = tabs[ti];
    memset(&d, 0, sizeof(d));
    d.dim = t.dim;
    Piece pc;
    const double ax0 = (t.role >= 1) ? kFromSIeV : 1.0;
    const double vf = t.role == 1 ? 1e-9 : t.role == 4 ? kFromSIeV : 1.0;
    for (int k = 0; k < t.dim; ++k) {
      d.n[k] = t.n[k];
      pc.offs.push_back(&d.off_x[k]);
      pc.rel.push_back((int)pc.data.size());
      const double f = k == 0 ? ax0 : 1.0;
      for (double v : t.x[k]) pc.data.push_back((R)(v * f));
      d.off_x64[k] = (int)dbl.size();
      for (double v : t.x[k]) dbl.push_back(v * f);
      d.domain[k][0] = t.domain[k][0] * f;
      d.domain[k][1] = t.domain[k][1] * f;
    }
    d.off_v64 = -1;
    if (t.dim == 3) {
      d.off_v64 = (int)dbl.size();
      for (double v : t.v) dbl.push_back(v * vf);
    }
    pc.offs.push_back(&d.off_v);
    pc.rel.push_back((int)pc.data.size());
    for (double v : t.v) pc.data.push_back((R)(v * vf));
    d.range[0] = t.range[0] * vf;
    d.range[1] = t.range[1] * vf;
    pieces.push_back(std::move(pc));
  }
  // NIST Mott elements
  std::vector<Mott> motts(ctx->mott.size());
  std::map<int, int> mottIndex;
  {
    size_t mi = 0;
    for (auto& kv : ctx->mott) {
      Mott& m = motts[mi];
      memset(&m, 0, sizeof(m));
      mott_constants(kv.first, kv.second, m);
      Piece pc;
      pc.offs.push_back(&m.off_spwem);
      pc.rel.push_back(0);
      for (double v : kv.second.spwem) pc.data.push_back((R)v);
      pieces.push_back(std::move(pc));
      m.off_x1 = -1;
      m.off_x1d = (int)dbl.size();  // the quantile table in double as well (the angle's cubic needs it)
      for (double v : kv.second.x1) dbl.push_back(v);
      mottIndex[kv.first] = (int)mi++;
    }
  }
  int nstage = 0;
  {
    std::vector<size_t> order(pieces.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return pieces[a].data.size() < pieces[b].data.size(); });
    const size_t align = 16 / sizeof(R);
    bool staging = true;
    for (size_t k : order) {
      Piece& pc = pieces[k];
      if (staging && (blob.size() + pc.data.size()) * sizeof(R) > kStageBytes) {
        staging = false;
        while (blob.size() % align) blob.push_back(R(0));
        nstage = (int)blob.size();
      }
      const int base = (int)blob.size();
      for (size_t f = 0; f < pc.offs.size(); ++f) *pc.offs[f] = base + pc.rel[f];
      blob.insert(blob.end(), pc.data.begin(), pc.data.end());
    }
    if (staging) {
      while (blob.size() % align) blob.push_back(R(0));
      nstage = (int)blob.size();
    }
  }
  // scatter models
  std::vector<Msm> msms;
  std::vector<Mech> mechs;
  for (auto& hm : ctx->msms) {
    const HMaterial& mt = ctx->mats[hm.material];
    Msm m;
    memset(&m, 0, sizeof(m));
    m.material = hm.material;
    m.vacuum = mt.Z.empty();
    double minE = m.vacuum ? -INFINITY : std::max(0.0, -mt.ecb);
    if (hm.minSet) minE = hm.minE;
    m.minE = minE * kFromSIeV;
    m.ecb = mt.ecb * kFromSIeV;
    m.u0 = mt.ecb * kFromSIeV;
    m.classical = hm.classical;
    m.lambda = hm.lambda * 1e9;
    m.lambdaFactor = (kPi * hm.lambda * sqrt(kElectronMass / 2.)) / kHbar * sqrt(kEV);
    m.csd = hm.csd;
    if (hm.csd) m.jln = make_jln(mt, hm.breakE);
    m.mech0 = (int)mechs.size();
    m.nmech = (int)hm.mechs.size();
    for (auto& hk : hm.mechs) {
      Mech k;
      memset(&k, 0, sizeof(k));
      k.kind = hk.kind;
      if (hk.kind == MECH_NISTMOTT) {
        k.nel = (int)mt.Z.size();
        const double densityNa = mt.density * kAvogadro;
        for (int i = 0; i < k.nel; ++i) {
          auto it = mottIndex.find(mt.Z[i]);
          if (it == mottIndex.end()) return fail(CM_ESTATE, "no NIST Mott table for Z=" + std::to_string(mt.Z[i]));
          k.mott[i] = it->second;
          k.mottMethod = hk.method;
          const double sf = (1000. * mt.wf[i]) / mt.A[i];
          k.kbrown[i] = sf * densityNa * 1e-9;
          k.kel[i] = (kBohr * kBohr) * sf * densityNa * 1e-9;
        }
      } else if (hk.kind == MECH_TABULATED) {
        k.methodSE = (hk.method != 2) && (hk.method != 3) ? 1 : hk.method;
        k.tIIMFP = hk.tables[0];
        k.tRed = hk.tables[1];
        k.tTheta = hk.tables[2];
        k.tSEE0 = hk.tables[3];
        k.energyOffset = hk.energyOffset * kFromSIeV;
        k.minEgenSE = 0.;
        k.rateMult = 1.;
        k.energyCBbottom = mt.ecb * kFromSIeV;
        k.bandgap = mt.bandgap * kFromSIeV;
        k.energyGap = k.bandgap;
        k.offsetFermiEnergy = (efermi(mt) + hk.energyOffset) * kFromSIeV;
        k.bEref = (mt.bandgap > 0. ? -mt.bandgap : efermi(mt)) * kFromSIeV;
        k.ncore = (int)mt.core.size();
        for (int i = 0; i < k.ncore && i < kMaxCore; ++i) k.core[i] = mt.core[i] * kFromSIeV;
        const Table& tr = tabs[k.tRed];
        const Table& tt = tabs[k.tTheta];
        k.eiDomain0 = std::max(tr.domain[0][0], tt.domain[0][0]);
        k.eiDomain1 = std::min(tr.domain[0][1], tt.domain[0][1]);
        k.iimfpDomain0 = tabs[k.tIIMFP].domain[0][0];
        if (k.methodSE >= 2) {
          k.rangeSE0lo = tabs[k.tSEE0].range[0];
          k.rangeSE0hi = tabs[k.tSEE0].range[1];
        }
      } else if (hk.kind == MECH_FITTED) {
        k.energySEgen = hk.energySEgen * kFromSIeV;
        k.eFermi = efermi(mt) * kFromSIeV;
        k.csd = make_jln(mt, hk.breakE);
      } else if (hk.kind == MECH_PHONON) {
        k.phononE = hk.phononE * kFromSIeV;
        double occ = 0.5 * (1. + (1. / (exp(hk.phononE / (kBoltzmann * hk.temperature)) - 1.)));
        double epsRatio = (hk.eps0 - hk.epsInf) / hk.eps0 / hk.epsInf;
        k.prefactor = (hk.ratemult * occ * epsRatio) / kBohr * 1e-9;
      } else if (hk.kind == MECH_POLARON) {
        k.prefactor = hk.prefactor * 1e-9;
        k.extinction = hk.extinction * kEV;
        k.cutoff = (-log(10. / hk.prefactor) / hk.extinction) * kFromSIeV;
      }
      mechs.push_back(k);
    }
    msms.push_back(m);
  }
  // geometry in nm
  std::vector<Shape> shapes;
  std::vector<Plane> planes;
  for (auto& hs : ctx->shapes) {
    Shape s;
    memset(&s, 0, sizeof(s));
    s.kind = hs.kind;
    s.a = hs.a;
    s.b = hs.b;
    for (int k = 0; k < 3; ++k) s.c[k] = hs.c[k] * 1e9;
    s.r = hs.r * 1e9;
    if (hs.kind == SHAPE_CYLINDER) {
      for (int k = 0; k < 3; ++k) {
        s.e0[k] = hs.e0[k] * 1e9;
        s.ax[k] = hs.ax[k] * 1e9;
        s.nax[k] = hs.nax[k];
      }
      s.rad2 = (hs.radius * 1e9) * (hs.radius * 1e9);
      s.len2 = (s.ax[0] * s.ax[0]) + (s.ax[1] * s.ax[1]) + (s.ax[2] * s.ax[2]);
      s.len = sqrt(s.len2);
    }
    if (hs.kind == SHAPE_PLANES) {
      s.plane0 = (int)planes.size();
      s.np = (int)hs.n.size() / 3;
      for (int i = 0; i < s.np; ++i) {
        Plane p;
        for (int k = 0; k < 3; ++k) {
          p.n[k] = hs.n[3 * i + k];
          p.p[k] = hs.p[3 * i + k] * 1e9;
        }
        planes.push_back(p);
      }
    }
    shapes.push_back(s);
  }
  // The batched (FP32) form merges every intersection of plane sets into one
  // plane set: an intersection of convex polytopes is the polytope bounded by
  // all their planes, so the first crossing and its normal are the same up to
  // rounding (and up to the reference's corner average when two children are
  // struck at exactly the same u), and the kernels need no tree walk.  The
  // plain (FP64) form keeps NormalIntersectionShape's march as written.
  if (sizeof(R) == 4 && !(ctx->options & CM_OPT_EXACT_CSG)) {
    for (size_t i = 0; i < shapes.size(); ++i) {
      if (shapes[i].kind != SHAPE_INTERSECTION) continue;
      std::vector<int> todo{(int)i}, leaves;
      while (!todo.empty()) {  // leaves in depth-first order, child a before child b
        const int id = todo.back();
        todo.pop_back();
        const HShape& hs = ctx->shapes[id];
        if (hs.kind == SHAPE_INTERSECTION) {
          todo.push_back(hs.b);
          todo.push_back(hs.a);
        } else {
          leaves.push_back(id);
        }
      }
      bool planar = true;
      for (int l : leaves) planar = planar && shapes[l].kind == SHAPE_PLANES;
      if (!planar) continue;
      const int plane0 = (int)planes.size();
      for (int l : leaves)
        for (int k = 0; k < shapes[l].np; ++k) {
          const Plane pl = planes[shapes[l].plane0 + k];
          planes.push_back(pl);
        }
      shapes[i].kind = SHAPE_PLANES;
      shapes[i].plane0 = plane0;
      shapes[i].np = (int)planes.size() - plane0;
    }
  }
  std::vector<int> sdepth(shapes.size(), 0);  // children come before their parents
  int depth = 0;
  for (size_t i = 0; i < shapes.size(); ++i) {
    Shape& sh = shapes[i];
    sh.anyunion = sh.kind == SHAPE_UNION;
    if (sh.kind == SHAPE_INTERSECTION || sh.kind == SHAPE_UNION) {
      sdepth[i] = 1 + std::max(sdepth[sh.a], sdepth[sh.b]);
      sh.anyunion = sh.anyunion || shapes[sh.a].anyunion || shapes[sh.b].anyunion;
    }
    depth = std::max(depth, sdepth[i]);
  }
  std::vector<Region> regions;
  std::vector<int> children;
  for (auto& hr : ctx->regions) {
    Region r;
    r.parent = hr.parent;
    r.msm = hr.msm;
    r.shape = hr.shape;
    r.child0 = (int)children.size();
    r.nchild = (int)hr.children.size();
    r.cls = hr.msm < kClasses ? hr.msm : kClasses - 1;
    // the box in nm, widened so that rounding never excludes a crossing or a point on the surface
    const Box bx = shape_box(ctx, hr.shape);
    for (int a = 0; a < 3; ++a) {
      const double pad = 1e-3 + 1e-9 * std::max(fabs(bx.lo[a]), fabs(bx.hi[a])) * 1e9;
      r.bb[a] = bx.lo[a] <= -kBoxWorld * 0.999 ? -INFINITY : bx.lo[a] * 1e9 - pad;
      r.bb[3 + a] = bx.hi[a] >= kBoxWorld * 0.999 ? INFINITY : bx.hi[a] * 1e9 + pad;
    }
    for (int c : hr.children) children.push_back(c);
    r.grid = -1;
    regions.push_back(r);
  }
  // grids over the children of regions with many of them (a rough-line layout: hundreds of segments)
  std::vector<ChildGrid> grids;
  std::vector<int> cell_start, grid_items;
  for (Region& r : regions) {
    if (r.nchild < kGridMinChildren || (ctx->options & CM_OPT_SCAN_CHILDREN)) continue;
    std::vector<int> bounded, unbounded;
    double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
    for (int i = 0; i < r.nchild; ++i) {
      const double* bb = regions[children[r.child0 + i]].bb;
      if (std::isinf(bb[0]) || std::isinf(bb[1]) || std::isinf(bb[3]) || std::isinf(bb[4]) || bb[0] > bb[3] ||
          bb[1] > bb[4]) {
        unbounded.push_back(i);
        continue;
      }
      bounded.push_back(i);
      for (int a = 0; a < 2; ++a) {
        lo[a] = std::min(lo[a], bb[a]);
        hi[a] = std::max(hi[a], bb[3 + a]);
      }
    }
    if ((int)bounded.size() < kGridMinChildren) continue;
    ChildGrid g;
    const double wx = std::max(hi[0] - lo[0], 1e-3), wy = std::max(hi[1] - lo[1], 1e-3);
    const double cells = std::min(65536.0, std::max(16.0, 2.0 * bounded.size()));
    g.nx = std::max(1, std::min(4096, (int)ceil(sqrt(cells * wx / wy))));
    g.ny = std::max(1, std::min(4096, (int)ceil(cells / g.nx)));
    g.x0 = lo[0];
    g.y0 = lo[1];
    g.dx = wx / g.nx;
    g.dy = wy / g.ny;
    std::vector<std::vector<int>> lists((size_t)g.nx * g.ny);
    for (int i : bounded) {  // ascending positions, so every cell list is ascending
      const double* bb = regions[children[r.child0 + i]].bb;
      const int ix0 = std::max(0, (int)floor((bb[0] - g.x0) / g.dx)), ix1 = std::min(g.nx - 1, (int)floor((bb[3] - g.x0) / g.dx));
      const int iy0 = std::max(0, (int)floor((bb[1] - g.y0) / g.dy)), iy1 = std::min(g.ny - 1, (int)floor((bb[4] - g.y0) / g.dy));
      for (int iy = iy0; iy <= iy1; ++iy)
        for (int ix = ix0; ix <= ix1; ++ix) lists[(size_t)iy * g.nx + ix].push_back(i);
    }
    g.cell0 = (int)cell_start.size();
    for (auto& l : lists) {
      cell_start.push_back((int)grid_items.size());
      grid_items.insert(grid_items.end(), l.begin(), l.end());
    }
    cell_start.push_back((int)grid_items.size());
    g.unb0 = (int)grid_items.size();
    g.nunb = (int)unbounded.size();
    grid_items.insert(grid_items.end(), unbounded.begin(), unbounded.end());
    r.grid = (int)grids.size();
    grids.push_back(g);
  }
  SceneView<R>& v = ds.view;
  int rc = 0;
  const bool h = ds.host;
  if ((rc = dev_copy(ds.allocs, shapes, &v.shapes, h)) || (rc = dev_copy(ds.allocs, planes, &v.planes, h)) ||
      (rc = dev_copy(ds.allocs, regions, &v.regions, h)) || (rc = dev_copy(ds.allocs, children, &v.children, h)) ||
      (rc = dev_copy(ds.allocs, msms, &v.msms, h)) || (rc = dev_copy(ds.allocs, mechs, &v.mechs, h)) ||
      (rc = dev_copy(ds.allocs, motts, &v.mott, h)) || (rc = dev_copy(ds.allocs, tabs, &v.tables, h)) ||
      (rc = dev_copy(ds.allocs, blob, &v.blob, h)) || (rc = dev_copy(ds.allocs, dbl, &v.dbl, h)) ||
      (rc = dev_copy(ds.allocs, grids, &v.grids, h)) || (rc = dev_copy(ds.allocs, cell_start, &v.cell_start, h)) ||
      (rc = dev_copy(ds.allocs, grid_items, &v.grid_items, h)))
    return rc;
  v.chamber = 0;
  v.options = ctx->options;
  v.depth = depth;
  v.dl50 = log(0.050 * kToSIkeV * kFromSIeV);
  v.param = (log(20.0 * kToSIkeV) - log(0.050 * kToSIkeV)) / 60.0;
  v.maxMott = 20.0 * kToSIkeV * kFromSIeV;
  v.nstaged = 0;
  v.nstage = nstage;
  ++ds.gen;
  ds.valid = true;
  return 0;
}

template <typename R> static DevScene<R>& scene_of(cm_context* c);
template <> DevScene<double>& scene_of<double>(cm_context* c) { return c->d64; }
template <> DevScene<float>& scene_of<float>(cm_context* c) { return c->d32; }
template <typename R> static RunBuffers<R>& buffers_of(cm_context* c);
template <> RunBuffers<double>& buffers_of<double>(cm_context* c) { return c->rb64; }
template <> RunBuffers<float>& buffers_of<float>(cm_context* c) { return c->rb32; }

// ------------------------------------------------------------------ kernels
// warp-aggregated append: one atomic per group of converged lanes
struct DeviceSink {
  __device__ __forceinline__ int append(int* counter) {
    cg::coalesced_group g = cg::coalesced_threads();
    int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(counter, (int)g.size());
    base = g.shfl(base, 0);
    return base + (int)g.thread_rank();
  }
  // lanes may target different counters (one per event queue): group them by
  // queue first, then one atomic per group
  __device__ __forceinline__ int append_q(int* counters, int q) {
    cg::coalesced_group g = cg::coalesced_threads();
    cg::coalesced_group part = cg::labeled_partition(g, q);
    int base = 0;
    if (part.thread_rank() == 0) base = atomicAdd(counters + q, (int)part.size());
    base = part.shfl(base, 0);
    return base + (int)part.thread_rank();
  }
  __device__ __forceinline__ void count(uint32_t* h) { atomicAdd(h, 1u); }
  // counters[idx] += value, one atomic per group of converged lanes with the same idx
  __device__ __forceinline__ void add_by(unsigned long long* counters, int idx, unsigned long long value) {
    cg::coalesced_group g = cg::coalesced_threads();
    cg::coalesced_group part = cg::labeled_partition(g, idx);
    const unsigned long long sum = cg::reduce(part, value, cg::plus<unsigned long long>());
    if (part.thread_rank() == 0) atomicAdd(counters + idx, sum);
  }
  __device__ __forceinline__ unsigned long long ticket(unsigned long long* c) { return atomicAdd(c, 1ull); }
  __device__ __forceinline__ void error(int* e, int code) { atomicExch(e, code); }
};

// The staged prefix of the table blob (v.s.nstaged elements, a multiple of 16 bytes, 16-byte aligned at
// both ends) into this block's shared memory: one bulk copy by the tensor memory accelerator completing on
// an mbarrier.  The wait is bounded; a copy that has not landed by then sets CM_ETIMEOUT and the block
// does no work (the host ends the run with that error).  Every thread of the block must call it.
template <typename R> __device__ __forceinline__ bool stage_tables(const RunView<R>& v) {
  const int n = v.s.nstaged;
  if (n <= 0) return true;
  __shared__ __align__(8) unsigned long long bar;
  const unsigned bar_a = (unsigned)__cvta_generic_to_shared(&bar);
  const unsigned dst = (unsigned)__cvta_generic_to_shared(cm_stage_smem);
  const unsigned bytes = (unsigned)n * (unsigned)sizeof(R);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(v.s.blob), "r"(bytes), "r"(bar_a)
                 : "memory");
  }
  unsigned done = 0;
  for (int it = 0; it < (1 << 20) && !done; ++it) {
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(bar_a)
        : "memory");
  }
  if (!done) atomicExch(&v.c->error, CM_ETIMEOUT);
  return __syncthreads_and(done) != 0;
}

__device__ __forceinline__ void flush_counts(Counters* c, StepCounts& sc) {
  for (int off = 16; off > 0; off >>= 1) {
    sc.steps += __shfl_down_sync(0xffffffffu, sc.steps, off);
    sc.scat += __shfl_down_sync(0xffffffffu, sc.scat, off);
    sc.bar += __shfl_down_sync(0xffffffffu, sc.bar, off);
    sc.esc += __shfl_down_sync(0xffffffffu, sc.esc, off);
    sc.sec += __shfl_down_sync(0xffffffffu, sc.sec, off);
    sc.zero += __shfl_down_sync(0xffffffffu, sc.zero, off);
    sc.limit += __shfl_down_sync(0xffffffffu, sc.limit, off);
  }
  if ((threadIdx.x & 31) == 0) {
    if (sc.steps) atomicAdd(&c->steps, sc.steps);
    if (sc.scat) atomicAdd(&c->scatters, sc.scat);
    if (sc.bar) atomicAdd(&c->barriers, sc.bar);
    if (sc.esc) atomicAdd(&c->escapes, sc.esc);
    if (sc.sec) atomicAdd(&c->secondaries, sc.sec);
    if (sc.zero) atomicAdd(&c->ended_zero, sc.zero);
    if (sc.limit) atomicAdd(&c->ended_limit, sc.limit);
  }
}

// Where each class segment of wave `cur` starts in the order the threads take its electrons, in the block's
// shared memory (a per-thread array indexed by segment would live in local memory).  Every thread of the
// block calls it.
__device__ __forceinline__ void segment_starts(const Counters* c, int cur, int* first) {
  if (threadIdx.x == 0) {
    int a = 0;
    for (int k = 0; k < kSegments; ++k) {
      first[k] = a;
      a += c->nc[cur][k];
    }
    first[kSegments] = a;
  }
  __syncthreads();
}

__device__ __forceinline__ int segment_of(const int* first, int i) {
  int k = 0;
  while (k < kSegments - 1 && i >= first[k + 1]) ++k;
  return k;
}

template <typename R, int D> __device__ __forceinline__ void flight_loop(const RunView<R>& v, int cur) {
  DeviceSink sink;
  StepCounts sc;
  const int n = v.c->n[cur];
  if ((int)(blockIdx.x * blockDim.x) >= n || !stage_tables(v)) return;  // blocks without work stage nothing
  __shared__ int first[kSegments + 1];
  segment_starts(v.c, cur, first);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = segment_of(first, i);  // the i-th electron over the class segments in order
    flight_one<R, D>(v, cur, k * v.W + (i - first[k]), sink, sc);
  }
  flush_counts(v.c, sc);
}

// FP64 flight: register-hungry double geometry and physics, compiled without an occupancy target
template <typename R, int D> __global__ void __launch_bounds__(256) k_flight(RunView<R> v, int cur) {
  flight_loop<R, D>(v, cur);
}

// Kernels that stage the small tables into shared memory (1 flight, 2 elastic, 4 inelastic, 8 steps) and
// the inelastic grid in blocks per SM when it stages.  k_inelastic gathers ~130 table values per event
// (cubic interpolation in the 2-D energy-loss and SE tables and the 3-D angle table); staged into the
// shared memory of a grid of 2 resident blocks per SM it gains 1 % on the linescan.  Staging in the
// other kernels, whose few small-table reads hit L1, loses 4 % (a copy per block, less L1).
#ifndef CM_STAGE_KERNELS
#define CM_STAGE_KERNELS 4
#endif
#ifndef CM_INEL_BLOCKS_PER_SM
#define CM_INEL_BLOCKS_PER_SM 2
#endif

// Resident CTAs per SM the kernels are compiled for (register caps 65536 / (256 x n)); a build may set
// them with -DCM_MINB_FLIGHT32=n and so on.  CM_MINB_INELASTIC unset: the compiler chooses.
#ifndef CM_MINB_FLIGHT32
#define CM_MINB_FLIGHT32 3
#endif
#ifndef CM_MINB_ELASTIC
#define CM_MINB_ELASTIC 4
#endif
#if defined(CM_MINB_ELASTIC)
#define CM_LB_ELASTIC __launch_bounds__(256, CM_MINB_ELASTIC)
#else
#define CM_LB_ELASTIC __launch_bounds__(256)
#endif
#if defined(CM_MINB_INELASTIC)
#define CM_LB_INELASTIC __launch_bounds__(256, CM_MINB_INELASTIC)
#else
#define CM_LB_INELASTIC __launch_bounds__(256)
#endif

// FP32 flight over leaf shapes compiled for 3 resident CTAs per SM (80 registers): the kernel is
// latency-bound and the extra warps hide more than the spills cost (linescan +5 %, rough image +3 %
// against 2 CTAs per SM; 4 CTAs spill twice as much and lose 7 % on the rough image).  Tree walks
// (D > 0) spill too much under a cap and keep k_flight.  k_elastic runs at 4 CTAs per SM (64
// registers, a few spills): linescan +2 %.
__global__ void __launch_bounds__(256, CM_MINB_FLIGHT32) k_flight32_leaf(RunView<float> v, int cur) {
  flight_loop<float, 0>(v, cur);
}

template <typename R>
__global__ void CM_LB_ELASTIC k_elastic(RunView<R> v, int cur) {
  DeviceSink sink;
  const int n = v.c->q[Q_EL];
  if ((int)(blockIdx.x * blockDim.x) >= n || !stage_tables(v)) return;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) elastic_one(v, cur, j, sink);
}

template <typename R>
__global__ void CM_LB_INELASTIC k_inelastic(RunView<R> v, int cur) {
  DeviceSink sink;
  StepCounts sc;
  const int n = v.c->q[Q_TAB];
  if ((int)(blockIdx.x * blockDim.x) >= n || !stage_tables(v)) return;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) inelastic_one(v, cur, j, sink, sc);
  flush_counts(v.c, sc);
}

template <typename R, int D>
__global__ void __launch_bounds__(256) k_misc(RunView<R> v, int cur) {
  DeviceSink sink;
  StepCounts sc;
  const int n = v.c->q[Q_MISC];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    misc_one<R, D>(v, cur, j, sink, sc);
  flush_counts(v.c, sc);
}

// the kernels are compiled for the intersection nestings 0 (leaf shapes only), 2 and 4
// smem: bytes of staged tables (v.s.nstaged elements), 0 when the view stages none
static void launch_flight(const RunView<double>& v, int cur, int grid, cudaStream_t s, size_t smem = 0) {
  if (v.s.depth == 0) k_flight<double, 0><<<grid, 256, smem, s>>>(v, cur);
  else if (v.s.depth <= 2) k_flight<double, 2><<<grid, 256, smem, s>>>(v, cur);
  else k_flight<double, kMaxShapeDepth><<<grid, 256, smem, s>>>(v, cur);
}

static void launch_flight(const RunView<float>& v, int cur, int grid, cudaStream_t s, size_t smem = 0) {
  if (v.s.depth == 0) k_flight32_leaf<<<grid, 256, smem, s>>>(v, cur);
  else if (v.s.depth <= 2) k_flight<float, 2><<<grid, 256, smem, s>>>(v, cur);
  else k_flight<float, kMaxShapeDepth><<<grid, 256, smem, s>>>(v, cur);
}

// The tail of a run: once fewer electrons are left than fill the GPU, each thread takes one electron
// through CM_TAIL_STEPS whole steps per iteration (k_steps) instead of one step through the queue
// kernels, whose launches and queue traffic then cost more than the steps themselves.
#ifndef CM_TAIL_BELOW
#define CM_TAIL_BELOW 262144
#endif
#ifndef CM_TAIL_STEPS
#define CM_TAIL_STEPS 32
#endif
#if defined(CM_MINB_STEPS)
#define CM_LB_STEPS __launch_bounds__(256, CM_MINB_STEPS)
#else
#define CM_LB_STEPS __launch_bounds__(256)
#endif

template <typename R, int D> __global__ void CM_LB_STEPS k_steps(RunView<R> v, int cur, int nsteps) {
  DeviceSink sink;
  StepCounts sc;
  const int n = v.c->n[cur];
  if ((int)(blockIdx.x * blockDim.x) >= n || !stage_tables(v)) return;
  __shared__ int first[kSegments + 1];
  segment_starts(v.c, cur, first);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = segment_of(first, i);
    steps_one<R, D>(v, cur, k * v.W + (i - first[k]), nsteps, sink, sc);
  }
  flush_counts(v.c, sc);
}

template <typename R>
static void launch_steps(const RunView<R>& v, int cur, int grid, int nsteps, cudaStream_t s, size_t smem) {
  if (v.s.depth == 0) k_steps<R, 0><<<grid, 256, smem, s>>>(v, cur, nsteps);
  else if (v.s.depth <= 2) k_steps<R, 2><<<grid, 256, smem, s>>>(v, cur, nsteps);
  else k_steps<R, kMaxShapeDepth><<<grid, 256, smem, s>>>(v, cur, nsteps);
}

// the launch settings a run uses: the context's tuning, built-in defaults where it holds 0
template <typename R> static cm_tuning resolved_tuning(const cm_context* ctx) {
  cm_tuning t = ctx->tune[sizeof(R) == 8 ? CM_PREC_FP64 : CM_PREC_FP32];
  if (t.wave <= 0) t.wave = 1 << 21;
  if (t.tail_below <= 0) t.tail_below = CM_TAIL_BELOW;
  if (t.tail_steps <= 0) t.tail_steps = CM_TAIL_STEPS;
  if (t.blocks_per_sm <= 0) t.blocks_per_sm = 8;
  return t;
}

template <typename R> static void launch_misc(const RunView<R>& v, int cur, int grid, cudaStream_t s) {
  if (v.s.depth == 0) k_misc<R, 0><<<grid, 256, 0, s>>>(v, cur);
  else if (v.s.depth <= 2) k_misc<R, 2><<<grid, 256, 0, s>>>(v, cur);
  else k_misc<R, kMaxShapeDepth><<<grid, 256, 0, s>>>(v, cur);
}

template <typename R, int D>
__global__ void __launch_bounds__(256) k_spawn(RunView<R> v, int cur) {
  const int nxt = cur ^ 1;
  int nn, take_se, take_p;
  refill_plan(v.c, nxt, v.W, v.poolCap, nn, take_se, take_p);
  const int poolTop = v.c->pool < v.poolCap ? v.c->pool : v.poolCap;
  const unsigned long long first = v.c->next_primary;
  DeviceSink sink;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < take_se + take_p; j += gridDim.x * blockDim.x)
    spawn_one<R, D>(v, nxt, j, take_se, poolTop, first, sink);
}

template <typename R> static void launch_spawn(const RunView<R>& v, int cur, int grid, cudaStream_t s) {
  if (v.s.depth == 0) k_spawn<R, 0><<<grid, 256, 0, s>>>(v, cur);
  else if (v.s.depth <= 2) k_spawn<R, 2><<<grid, 256, 0, s>>>(v, cur);
  else k_spawn<R, kMaxShapeDepth><<<grid, 256, 0, s>>>(v, cur);
}

template <typename R>
__global__ void k_tail(RunView<R> v, int cur, int steps) {
  if (blockIdx.x == 0 && threadIdx.x == 0) tail_update(v.c, cur, v.W, v.poolCap, steps != 0);
}

// The device-driven loop: each of its iterations ends with k_loop, which updates the counters as k_tail
// does and then sets the condition of the conditional node it runs under: another iteration, or not when
// the run is done or failed (a device error, the iteration limit, a cancel flag set by the host), and for
// the queue loop also once every primary has started and fewer electrons are left than io.tail_below
// (the tail loop of whole steps per thread takes over).  Iterations of a loop body after its end do no
// work: their kernels find no electrons.
template <typename R>
__global__ void k_loop(RunView<R> v, int cur, int steps, cudaGraphConditionalHandle h) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  Counters* c = v.c;
  tail_update(c, cur, v.W, v.poolCap, steps != 0);
  const RunIO& io = *v.io;
  c->slots += 1;
  if (steps) c->tail_slots += 1;
  if (!c->done && !c->error) {
    if ((long long)c->slots >= io.max_slots) c->error = CM_ELIMIT;
    else if (io.cancel && *io.cancel) c->error = CM_ECANCELED;
  }
  bool go = !c->done && !c->error;
  if (go && !steps && !io.queue_only) {
    const long long left = (long long)c->n[cur ^ 1] + (c->pool < v.poolCap ? c->pool : v.poolCap);
    if (c->next_primary == c->total_primaries && left < io.tail_below) go = false;
  }
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// opens a loop of the device-driven run unless the run is already done or failed
__global__ void k_gate(const Counters* c, cudaGraphConditionalHandle h) {
  if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, (!c->done && !c->error) ? 1u : 0u);
}

#ifdef CM_TRACE
static TraceRec* g_trace = nullptr;
static int* g_ntrace = nullptr;
static int g_tracecap = 0;
#endif

// One device buffer of the run: CM_ENOMEM when the device has no room (the runtime's error state is
// cleared, so the context stays usable and a smaller request can follow), CM_ECUDA for other failures.
static int run_alloc(std::vector<void*>& allocs, void** p, size_t bytes) {
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    char msg[128];
    snprintf(msg, sizeof(msg), "device memory exhausted allocating %zu bytes of run buffers", bytes);
    return fail(CM_ENOMEM, msg);
  }
  if (e != cudaSuccess) return fail(CM_ECUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  allocs.push_back(*p);
  return 0;
}

template <typename R>
static int alloc_wave(std::vector<void*>& allocs, Wave<R>& w, int cap) {
  auto A = [&](void** p, size_t bytes) -> int { return run_alloc(allocs, p, bytes); };
  int rc = 0;
  size_t n = (size_t)cap;
  if ((rc = A((void**)&w.px, n * 8)) || (rc = A((void**)&w.py, n * 8)) || (rc = A((void**)&w.pz, n * 8)) ||
      (rc = A((void**)&w.dx, n * sizeof(R))) || (rc = A((void**)&w.dy, n * sizeof(R))) ||
      (rc = A((void**)&w.dz, n * sizeof(R))) || (rc = A((void**)&w.E, n * sizeof(R))) ||
      (rc = A((void**)&w.Ep, n * sizeof(R))) || (rc = A((void**)&w.region, n * 4)) ||
      (rc = A((void**)&w.pixel, n * 4)) || (rc = A((void**)&w.aux, n * 4)) || (rc = A((void**)&w.step, n * 4)) ||
      (rc = A((void**)&w.key, n * 8)) || (rc = A((void**)&w.hx, n * sizeof(R))) ||
      (rc = A((void**)&w.hy, n * sizeof(R))) || (rc = A((void**)&w.hz, n * sizeof(R))))
    return rc;
  return 0;
}

// bytes of one electron record (Wave<R>): position 3 x f64, 8 fields of R, 4 int32, the u64 key
template <typename R> constexpr size_t record_bytes() { return 3 * 8 + 8 * sizeof(R) + 4 * 4 + 8; }

template <typename R>
static int ensure_buffers(cm_context* ctx, int W, int poolCap) {
  RunBuffers<R>& rb = buffers_of<R>(ctx);
  if (rb.cap == W && rb.poolCap >= poolCap) return 0;
  NvtxRange range("cm run buffers");
  rb.release();
  // two waves of kSegments segments, the pool, three queues: refused before any allocation when the
  // device has not that much free memory (less a reserve for the run's other buffers)
  const size_t need = ((size_t)2 * kSegments * W + (size_t)poolCap) * record_bytes<R>() + (size_t)3 * W * 4;
  size_t freeb = 0, totalb = 0;
  CM_CUDA(cudaMemGetInfo(&freeb, &totalb));
  if (need + ((size_t)256 << 20) > freeb) {
    char msg[160];
    snprintf(msg, sizeof(msg), "a wave of %d electrons needs %.1f GB of run buffers, %.1f GB are free", W,
             need / 1e9, freeb / 1e9);
    return fail(CM_ENOMEM, msg);
  }
  int rc;
  if ((rc = alloc_wave(rb.allocs, rb.w[0], kSegments * W)) || (rc = alloc_wave(rb.allocs, rb.w[1], kSegments * W)) ||
      (rc = alloc_wave(rb.allocs, rb.pool, poolCap))) {
    rb.release();  // nothing half-built stays behind: the next run allocates afresh
    return rc;
  }
  for (int k = 0; k < 3; ++k) {
    void* p;
    if ((rc = run_alloc(rb.allocs, &p, (size_t)W * 4))) {
      rb.release();
      return rc;
    }
    rb.q[k] = (int*)p;
  }
  if ((rc = run_alloc(rb.allocs, (void**)&rb.io, sizeof(RunIO)))) {
    rb.release();
    return rc;
  }
  rb.cap = W;
  rb.poolCap = poolCap;
  return 0;
}

// Secondary-pool records for a wave of W electrons and beams of up to emax_eV.  A wave full of primaries
// creates about one tracked secondary per 20 eV of their energy before it drains (the refill takes new
// primaries only into an empty pool), so the pool grows with the beam energy: 8 W at 1 keV and below, up
// to 64 W (factor > 0: factor W).  What this does not cover, the overflow restart does (it doubles the pool).
static int pool_records(int W, double emax_eV, int factor) {
  const double f = factor > 0 ? (double)factor : std::min(64.0, std::max(8.0, 8.0 * emax_eV / 1000.0));
  return (int)std::min<double>(f * (double)W, (double)(1 << 30));
}

// iterations of a loop body (an even number: the waves alternate)
constexpr int kLoopBody = 16;

// the kernels of one transport iteration of the queue loop and of the tail loop, launched on s
template <typename R>
static void launch_queue_iteration(const cm_context* ctx, const RunView<R>& v, const RunView<R>& vs, int cur, int grid,
                                   size_t smem, cudaStream_t s, cudaGraphConditionalHandle* h, cudaEvent_t* ev) {
  if (CM_STAGE_KERNELS & 1) launch_flight(vs, cur, grid, s, smem);
  else launch_flight(v, cur, grid, s);
  if (ev) cudaEventRecordWithFlags(ev[0], s, cudaEventRecordExternal);
  if (CM_STAGE_KERNELS & 2) k_elastic<R><<<grid, 256, smem, s>>>(vs, cur);
  else k_elastic<R><<<grid, 256, 0, s>>>(v, cur);
  if (ev) cudaEventRecordWithFlags(ev[1], s, cudaEventRecordExternal);
  if (CM_STAGE_KERNELS & 4) k_inelastic<R><<<ctx->nsm * CM_INEL_BLOCKS_PER_SM, 256, smem, s>>>(vs, cur);
  else k_inelastic<R><<<grid, 256, 0, s>>>(v, cur);
  if (ev) cudaEventRecordWithFlags(ev[2], s, cudaEventRecordExternal);
  launch_misc<R>(v, cur, grid, s);
  if (ev) cudaEventRecordWithFlags(ev[3], s, cudaEventRecordExternal);
  launch_spawn<R>(v, cur, grid, s);
  if (ev) cudaEventRecordWithFlags(ev[4], s, cudaEventRecordExternal);
  if (h) k_loop<R><<<1, 32, 0, s>>>(v, cur, 0, *h);
  else k_tail<R><<<1, 32, 0, s>>>(v, cur, 0);
  if (ev) cudaEventRecordWithFlags(ev[5], s, cudaEventRecordExternal);
}

template <typename R>
static void launch_tail_iteration(const RunView<R>& v, const RunView<R>& vs, int cur, int grid, int tail_steps,
                                  size_t smem, cudaStream_t s, cudaGraphConditionalHandle* h, cudaEvent_t* ev) {
  if (CM_STAGE_KERNELS & 8) launch_steps(vs, cur, grid, tail_steps, s, smem);
  else launch_steps(v, cur, grid, tail_steps, s, 0);
  if (ev) cudaEventRecordWithFlags(ev[0], s, cudaEventRecordExternal);
  launch_spawn<R>(v, cur, grid, s);
  if (ev) cudaEventRecordWithFlags(ev[1], s, cudaEventRecordExternal);
  if (h) k_loop<R><<<1, 32, 0, s>>>(v, cur, 1, *h);
  else k_tail<R><<<1, 32, 0, s>>>(v, cur, 1);
  if (ev) cudaEventRecordWithFlags(ev[2], s, cudaEventRecordExternal);
}

// One graph for a whole run: a gate, a WHILE loop of queue iterations, a gate, a WHILE loop of tail
// iterations (CUDA conditional nodes; k_loop decides on the device whether a loop goes on).  Its kernels
// read the run's inputs through v.io, so the instantiated graph is kept in the buffers and serves every
// later run with the same key; the host launches it once per run and reads the counters once.
template <typename R>
static int build_loop_graph(cm_context* ctx, RunBuffers<R>& rb, const RunView<R>& v, const RunView<R>& vs, int grid,
                            size_t smem, int tail_steps) {
  NvtxRange range("cm launch graph");
  rb.drop_graph();
  cudaGraph_t g = nullptr;
  CM_CUDA(cudaGraphCreate(&g, 0));
  auto bail = [&](cudaError_t e, const char* what) -> int {
    cudaGraphDestroy(g);
    return fail(CM_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  cudaError_t e;
  cudaGraphConditionalHandle h[2];
  for (int k = 0; k < 2; ++k)
    if ((e = cudaGraphConditionalHandleCreate(&h[k], g, 0, cudaGraphCondAssignDefault)) != cudaSuccess)
      return bail(e, "cudaGraphConditionalHandleCreate");
  cudaGraphNode_t prev = nullptr;
  for (int loop = 0; loop < 2; ++loop) {
    // the gate kernel, then the WHILE node whose body holds kLoopBody iterations
    const Counters* cp = v.c;
    cudaGraphConditionalHandle hh = h[loop];
    void* args[] = {(void*)&cp, (void*)&hh};
    cudaKernelNodeParams kp = {};
    kp.func = (void*)k_gate;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = args;
    cudaGraphNode_t gate, wnode;
    if ((e = cudaGraphAddKernelNode(&gate, g, prev ? &prev : nullptr, prev ? 1 : 0, &kp)) != cudaSuccess)
      return bail(e, "cudaGraphAddKernelNode");
    cudaGraphNodeParams cp2 = {};
    cp2.type = cudaGraphNodeTypeConditional;
    cp2.conditional.handle = hh;
    cp2.conditional.type = cudaGraphCondTypeWhile;
    cp2.conditional.size = 1;
    if ((e = cudaGraphAddNode(&wnode, g, &gate, 1, &cp2)) != cudaSuccess) return bail(e, "cudaGraphAddNode");
    cudaGraph_t body = cp2.conditional.phGraph_out[0];
    if ((e = cudaStreamBeginCaptureToGraph(ctx->cap_stream, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return bail(e, "cudaStreamBeginCaptureToGraph");
    for (int it = 0; it < kLoopBody; ++it) {
      if (loop == 0) launch_queue_iteration<R>(ctx, v, vs, it & 1, grid, smem, ctx->cap_stream, &hh, nullptr);
      else launch_tail_iteration<R>(v, vs, it & 1, grid, tail_steps, smem, ctx->cap_stream, &hh, nullptr);
    }
    cudaGraph_t captured = nullptr;
    if ((e = cudaStreamEndCapture(ctx->cap_stream, &captured)) != cudaSuccess) return bail(e, "cudaStreamEndCapture");
    prev = wnode;
  }
  cudaGraphExec_t exec = nullptr;
  if ((e = cudaGraphInstantiate(&exec, g, 0)) != cudaSuccess) return bail(e, "cudaGraphInstantiate");
  rb.loop_graph = g;
  rb.loop_exec = exec;
  return 0;
}

// the message of a device-side error code of a run
static int run_error(int err, const Counters& hc) {
  switch (err) {
    case CM_ETIMEOUT: return fail(err, "a table copy into shared memory did not complete in time");
    case CM_EOVERFLOW: return fail(err, "secondary pool overflow; raise the wave size");
    case CM_ECANCELED: return fail(err, "cancelled");
    case CM_ELIMIT: {
      char msg[256];
      snprintf(msg, sizeof(msg), "iteration limit reached (live %d %d, pool %d, primaries %llu of %llu)", hc.n[0],
               hc.n[1], hc.pool, hc.next_primary, hc.total_primaries);
      return fail(err, msg);
    }
    default: return fail(err, "the transport kernels reported error " + std::to_string(err));
  }
}

// print a few of the electrons still alive after an iteration limit (CM_DEBUG_DUMP set)
template <typename R> static void dump_live(const RunBuffers<R>& rb, const Counters& hc) {
  if (!getenv("CM_DEBUG_DUMP")) return;
  const int cur = hc.n[0] ? 0 : 1;
  const int k = std::min(8, hc.n[cur]);
  std::vector<double> px(k), py(k), pz(k);
  std::vector<R> E(k), dz(k);
  std::vector<int> reg(k);
  std::vector<uint32_t> stp(k);
  cudaMemcpy(px.data(), rb.w[cur].px, k * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(py.data(), rb.w[cur].py, k * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(pz.data(), rb.w[cur].pz, k * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(E.data(), rb.w[cur].E, k * sizeof(R), cudaMemcpyDeviceToHost);
  cudaMemcpy(dz.data(), rb.w[cur].dz, k * sizeof(R), cudaMemcpyDeviceToHost);
  cudaMemcpy(reg.data(), rb.w[cur].region, k * 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(stp.data(), rb.w[cur].step, k * 4, cudaMemcpyDeviceToHost);
  for (int i = 0; i < k; ++i)
    fprintf(stderr, "live[%d] pos %g %g %g nm E %g eV dz %g region %d step %u\n", i, px[i], py[i], pz[i], (double)E[i],
            (double)dz[i], reg[i], stp[i]);
}

// Transport loop.  Inputs are device arrays.  A run launches the cached device-driven loop graph once; a
// profiled run (d->profile) replays iterations from the host instead, with CUDA events between the kernels.
template <typename R>
static int run_device_once(cm_context* ctx, const cm_run_desc* d, uint32_t* back, uint32_t* fwd, cm_run_stats* st,
                      cudaStream_t stream, const unsigned long long* prefix_dev, const double* e0ref_dev,
                      const unsigned long long* pkey_dev, unsigned long long total, double emax_eV) {
  int rc;
  DevScene<R>& ds = scene_of<R>(ctx);
  if ((rc = build_scene<R>(ctx, ds))) return rc;
  const cm_tuning tu = resolved_tuning<R>(ctx);
  const int W = d->wave > 0 ? d->wave : tu.wave;
  RunBuffers<R>& rb0 = buffers_of<R>(ctx);
  const int poolWant = std::max(pool_records(W, emax_eV, tu.pool), rb0.cap == W ? rb0.poolCap : 0);
  if ((rc = ensure_buffers<R>(ctx, W, poolWant))) {
    // a pool sized for the beam energy that the device cannot hold: the smallest one (restarts grow it)
    if (rc != CM_ENOMEM || poolWant <= 8 * W || (rc = ensure_buffers<R>(ctx, W, 8 * W))) return rc;
  }
  RunBuffers<R>& rb = buffers_of<R>(ctx);
  RunView<R> v;
#ifdef CM_TRACE
  v.trace = g_trace;
  v.ntrace = g_ntrace;
  v.tracecap = g_tracecap;
#endif
  v.s = ds.view;
  v.s.chamber = d->chamber;
  v.w[0] = rb.w[0];
  v.w[1] = rb.w[1];
  v.pool = rb.pool;
  for (int k = 0; k < 3; ++k) v.q[k] = rb.q[k];
  v.c = ctx->counters;
  v.W = W;
  v.poolCap = rb.poolCap;
  v.io = rb.io;
  const int maxIt = d->max_iterations > 0 ? d->max_iterations : 500000;
  RunIO& io = *ctx->io_host;
  memset(&io, 0, sizeof(io));
  io.pc = d->pixel_center;
  io.pe0 = d->pixel_energy;
  io.pe0ref = e0ref_dev;
  io.pnbins = d->pixel_nbins;
  io.prefix = prefix_dev;
  io.npix = d->npix;
  io.width = d->beam_width * 1e9;  // m -> nm
  io.pkey = pkey_dev;
  io.pfirst = (const unsigned long long*)d->pixel_first;
  io.back = back;
  io.fwd = fwd;
  io.stride = d->hist_stride;
  io.elev = d->elevation && d->azimuth ? d->elevation : nullptr;
  io.azim = io.elev ? d->azimuth : nullptr;
  io.log = d->escape_log && d->escape_log_cap > 0 ? d->escape_log : nullptr;
  io.logCap = io.log ? d->escape_log_cap : 0;
  io.max_slots = maxIt;
  io.tail_below = tu.tail_below;
  io.queue_only = (ctx->options & CM_OPT_QUEUE_STEPS) ? 1 : 0;
  io.cancel = ctx->cancel ? ctx->cancel_dev : nullptr;
  CM_CUDA(cudaMemcpyAsync(rb.io, &io, sizeof(RunIO), cudaMemcpyHostToDevice, stream));

  Counters c0;
  memset(&c0, 0, sizeof(c0));
  c0.total_primaries = total;
  CM_CUDA(cudaMemcpyAsync(ctx->counters, &c0, sizeof(c0), cudaMemcpyHostToDevice, stream));
  const int grid = ctx->nsm * tu.blocks_per_sm;
  // the kernels that read tables (flight, elastic, inelastic, steps) stage the blob's small-table prefix
  // into shared memory unless CM_OPT_GLOBAL_TABLES; the others get a view without it
  v.s.nstaged = 0;
  RunView<R> vs = v;
  if (!(ctx->options & CM_OPT_GLOBAL_TABLES)) vs.s.nstaged = v.s.nstage;
  const size_t smem = (size_t)vs.s.nstaged * sizeof(R);
  cudaEvent_t e0, e1;
  CM_CUDA(cudaEventCreate(&e0));
  CM_CUDA(cudaEventCreate(&e1));
  double kms[6] = {0, 0, 0, 0, 0, 0};
  double step_ms = 0;
  long long qslots = 0, tslots = 0;
  int status = 0;
  if (!d->profile) {
    const LoopKey key{ds.gen, d->chamber, grid, ctx->nsm * CM_INEL_BLOCKS_PER_SM, tu.tail_steps, (int)vs.s.nstaged};
    if (!rb.loop_exec || !(rb.loop_key == key)) {
      if ((rc = build_loop_graph<R>(ctx, rb, v, vs, grid, smem, tu.tail_steps))) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
      }
      rb.loop_key = key;
    }
    CM_CUDA(cudaEventRecord(e0, stream));
    CM_CUDA(cudaGraphLaunch(rb.loop_exec, stream));
    CM_CUDA(cudaEventRecord(e1, stream));
    CM_CUDA(cudaMemcpyAsync(ctx->counters_host, ctx->counters, sizeof(Counters), cudaMemcpyDeviceToHost, stream));
    CM_CUDA(cudaStreamSynchronize(stream));
    const Counters& hc = *ctx->counters_host;
    tslots = (long long)hc.tail_slots;
    qslots = (long long)hc.slots - tslots;
    if (hc.error) {
      status = run_error(hc.error, hc);
      if (hc.error == CM_ELIMIT) dump_live(rb, hc);
    }
  } else {
    // profiled: the host replays captured iterations (events between the kernels) and reads the
    // counters after each replay
    const int K = kLoopBody;
    std::vector<cudaEvent_t> pev((size_t)K * 6 + 1), tev((size_t)K * 3 + 1);
    for (auto& ev : pev) CM_CUDA(cudaEventCreate(&ev));
    for (auto& ev : tev) CM_CUDA(cudaEventCreate(&ev));
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    for (int loop = 0; loop < 2; ++loop) {
      CM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      std::vector<cudaEvent_t>& ev = loop == 0 ? pev : tev;
      cudaEventRecordWithFlags(ev[0], stream, cudaEventRecordExternal);
      for (int it = 0; it < K; ++it) {
        if (loop == 0) launch_queue_iteration<R>(ctx, v, vs, it & 1, grid, smem, stream, nullptr, &pev[(size_t)it * 6 + 1]);
        else launch_tail_iteration<R>(v, vs, it & 1, grid, tu.tail_steps, smem, stream, nullptr, &tev[(size_t)it * 3 + 1]);
      }
      CM_CUDA(cudaStreamEndCapture(stream, &graph[loop]));
      CM_CUDA(cudaGraphInstantiate(&exec[loop], graph[loop], 0));
    }
    bool tail = false;
    CM_CUDA(cudaEventRecord(e0, stream));
    for (;;) {
      CM_CUDA(cudaGraphLaunch(exec[tail ? 1 : 0], stream));
      (tail ? tslots : qslots) += K;
      CM_CUDA(cudaMemcpyAsync(ctx->counters_host, ctx->counters, sizeof(Counters), cudaMemcpyDeviceToHost, stream));
      CM_CUDA(cudaStreamSynchronize(stream));
      for (int it = 0; it < K; ++it) {
        float ms[6] = {0, 0, 0, 0, 0, 0};
        if (!tail) {
          for (int k = 0; k < 6; ++k) cudaEventElapsedTime(&ms[k], pev[(size_t)it * 6 + k], pev[(size_t)it * 6 + k + 1]);
          for (int k = 0; k < 6; ++k) kms[k] += ms[k];
        } else {
          for (int k = 0; k < 3; ++k) cudaEventElapsedTime(&ms[k], tev[(size_t)it * 3 + k], tev[(size_t)it * 3 + k + 1]);
          step_ms += ms[0];
          kms[CM_K_SPAWN] += ms[1];
          kms[CM_K_TAIL] += ms[2];
        }
      }
      const Counters& hc = *ctx->counters_host;
      if (hc.error) {
        status = run_error(hc.error, hc);
        break;
      }
      if (hc.done) break;
      if (ctx->cancel && ctx->cancel->load()) {
        status = fail(CM_ECANCELED, "cancelled");
        break;
      }
      // all primaries started and fewer electrons left (waves and pool) than the tail threshold: the tail
      // iterations (unless CM_OPT_QUEUE_STEPS keeps the queue kernels to the end)
      const long long left = (long long)hc.n[0] + hc.n[1] + std::min(hc.pool, v.poolCap);
      tail = !(ctx->options & CM_OPT_QUEUE_STEPS) && hc.next_primary == hc.total_primaries && left < tu.tail_below;
      if (qslots + tslots >= maxIt) {
        status = run_error(CM_ELIMIT, hc);
        dump_live(rb, hc);
        break;
      }
    }
    CM_CUDA(cudaEventRecord(e1, stream));
    for (int loop = 0; loop < 2; ++loop) {
      cudaGraphExecDestroy(exec[loop]);
      cudaGraphDestroy(graph[loop]);
    }
    for (auto& ev : pev) cudaEventDestroy(ev);
    for (auto& ev : tev) cudaEventDestroy(ev);
  }
  CM_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CM_CUDA(cudaGetLastError());
  if (st) {
    const Counters& c = *ctx->counters_host;
    st->primaries = (int64_t)c.next_primary;
    st->steps = (int64_t)c.steps;
    st->scatter_events = (int64_t)c.scatters;
    st->barrier_events = (int64_t)c.barriers;
    st->escapes = (int64_t)c.escapes;
    st->secondaries = (int64_t)c.secondaries;
    st->iterations = (int64_t)c.iterations;
    st->device_ms = ms;
    for (int k = 0; k < 6; ++k) {
      st->kernel_ms[k] = kms[k];
      st->kernel_launches[k] = (int64_t)(k < 4 ? qslots : qslots + tslots);
    }
    for (int k = 0; k < 4; ++k) st->units[k] = (int64_t)c.units[k];
    st->step_launches = tslots;
    st->step_units = (int64_t)c.step_units;
    st->step_ms = step_ms;
    st->ended_zero_energy = (int64_t)c.ended_zero;
    st->ended_step_limit = (int64_t)c.ended_limit;
  }
  return status;
}

// zero the angle histograms a run tallies into (device arrays)
static int clear_angles(const cm_run_desc* d, cudaStream_t s) {
  if (!d->elevation || !d->azimuth) return 0;
  CM_CUDA(cudaMemsetAsync(d->elevation, 0, (size_t)d->npix * CM_ELEVATION_COUNTS * sizeof(uint32_t), s));
  CM_CUDA(cudaMemsetAsync(d->azimuth, 0, (size_t)d->npix * CM_AZIMUTH_COUNTS * sizeof(uint32_t), s));
  return 0;
}

// Every electron's random stream is keyed by its lineage, so a run that
// overflowed the secondary pool is repeated with a larger pool and gives the
// same tallies it would have given the first time.
template <typename R>
static int run_device(cm_context* ctx, const cm_run_desc* d, uint32_t* back, uint32_t* fwd, cm_run_stats* st,
                      cudaStream_t stream, const unsigned long long* prefix_dev, const double* e0ref_dev,
                      const unsigned long long* pkey_dev, unsigned long long total, double emax_eV) {
  const size_t hbytes = (size_t)d->npix * d->hist_stride * sizeof(uint32_t);
  int rc_clear;
  for (int attempt = 0;; ++attempt) {
    const int rc =
        run_device_once<R>(ctx, d, back, fwd, st, stream, prefix_dev, e0ref_dev, pkey_dev, total, emax_eV);
    if (st) st->pool_restarts = attempt;
    if (rc != CM_EOVERFLOW) return rc;
    RunBuffers<R>& rb = buffers_of<R>(ctx);
    const int W = rb.cap;
    const long long want = 2LL * rb.poolCap;
    if (want > (1LL << 30)) return rc;
    int e;
    if ((e = ensure_buffers<R>(ctx, W, (int)want))) return e;
    CM_CUDA(cudaMemsetAsync(back, 0, hbytes, stream));
    CM_CUDA(cudaMemsetAsync(fwd, 0, hbytes, stream));
    if ((rc_clear = clear_angles(d, stream))) return rc_clear;
  }
}

// ------------------------------------------------------------------ per-function kernels
template <typename R> __global__ void k_eval_nistmott(SceneView<R> s, int mi, int method, int n, const double* E, const double* u,
                                                      double* sig, double* th) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Mott& m = s.mott[mi];
  const R e = (R)(E[i] * kFromSIeV);
  // cross section in m^2 (rate factor 1/kbrown folded back): kel = a0^2, kbrown = 1
  sig[i] = (double)nistmott_rate(s, m, method, (R)(kBohr * kBohr), R(1), e, mlog(e));
  FixedRng<R> g{u + 2 * i, 2, 0};
  th[i] = (double)nistmott_angle(s, m, method, e, g);
}

template <typename R> __global__ void k_eval_table(SceneView<R> s, int t, int n, const double* x, double f0, double vf, int order,
                                                   double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = (double)table_interp(s, t, (R)(x[3 * i] * f0), (R)x[3 * i + 1], (R)x[3 * i + 2], order) / vf;
}

template <typename R> __global__ void k_eval_locate(SceneView<R> s, int t, int n, const double* x, double f0, int order,
                                                    double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int w[6];
  table_windows(s, t, (R)(x[3 * i] * f0), (R)x[3 * i + 1], (R)x[3 * i + 2], order, w);
  for (int k = 0; k < 6; ++k) out[6 * i + k] = w[k];
}

template <typename R> __global__ void k_eval_pick(SceneView<R> s, int msm, int n, const double* in, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Msm& m = s.msms[msm];
  const R E = (R)(in[2 * i] * kFromSIeV);
  R cum[kMaxMech];
  const R total = msm_cumulative_rates(s, m, E, cum);
  out[2 * i] = total != R(0) ? mech_pick(cum, m.nmech, (R)in[2 * i + 1] * total) : -1;
  out[2 * i + 1] = (double)total * 1e9;
}

template <typename R> __global__ void k_eval_tabulated(SceneView<R> s, int mech, int n, const double* in, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Mech& k = s.mechs[mech];
  const double* q = in + 9 * i;
  double* o = out + 12 * i;
  R E = (R)(q[0] * kFromSIeV);
  R d[3];
  dir_from_angles(d, (R)q[1], (R)q[2]);
  o[0] = (double)tabulated_rate(s, k, E) * 1e9;
  FixedRng<R> g{q + 3, 6, 0};
  R sd[3] = {0, 0, 0}, sE = 0, th = 0;
  const bool made = tabulated_scatter(s, k, d, E, sd, sE, g, &th);
  o[1] = (double)E * kEV;
  o[2] = d[0]; o[3] = d[1]; o[4] = d[2];
  o[5] = made;
  o[6] = made ? (double)sE * kEV : 0.;
  o[7] = sd[0]; o[8] = sd[1]; o[9] = sd[2];
  o[10] = g.used;
  o[11] = th;
}

template <typename R> __global__ void k_eval_elastic(SceneView<R> s, int mech, int n, const double* in, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Mech& k = s.mechs[mech];
  const double* q = in + 7 * i;
  double* o = out + 6 * i;
  const R E = (R)(q[0] * kFromSIeV);
  R d[3];
  dir_from_angles(d, (R)q[1], (R)q[2]);
  o[0] = (double)mech_rate(s, k, E, mlog(E)) * 1e9;
  FixedRng<R> g{q + 3, 4, 0};
  const int el = elastic_scatter(s, k, d, E, g);
  o[1] = d[0]; o[2] = d[1]; o[3] = d[2];
  o[4] = s.mott[k.mott[el]].Z;
  o[5] = g.used;
}

template <typename R> __global__ void k_eval_csd(SceneView<R> s, int msm, int n, const double* in, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Msm& m = s.msms[msm];
  const R E = (R)(in[2 * i] * kFromSIeV);
  const R len = (R)(in[2 * i + 1] * 1e9);
  out[3 * i] = m.csd ? (double)jln_compute(m.jln, len, E) * kEV : 0.;
  double fr = 0, pr = 0;
  for (int k = 0; k < m.nmech; ++k) {
    const Mech& mk = s.mechs[m.mech0 + k];
    if (mk.kind == MECH_FITTED) fr = (double)mech_rate(s, mk, E, mlog(E)) * 1e9;
    if (mk.kind == MECH_POLARON) pr = (double)mech_rate(s, mk, E, mlog(E)) * 1e9;
  }
  out[3 * i + 1] = fr;
  out[3 * i + 2] = pr;
}

template <typename R> __global__ void k_eval_phonon(SceneView<R> s, int mech, int n, const double* in, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Mech& k = s.mechs[mech];
  const double* q = in + 5 * i;
  double* o = out + 6 * i;
  R E = (R)(q[0] * kFromSIeV), Ep = E;
  R d[3];
  dir_from_angles(d, (R)q[1], (R)q[2]);
  o[0] = (double)phonon_rate(k, E) * 1e9;
  FixedRng<R> g{q + 3, 2, 0};
  phonon_scatter(k, d, E, Ep, g);
  o[1] = (double)E * kEV;
  o[2] = d[0]; o[3] = d[1]; o[4] = d[2];
  o[5] = (double)Ep * kEV;
}

__global__ void k_eval_shape(SceneView<double> s, int shape, int n, const double* p01, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double p0[3] = {p01[6 * i] * 1e9, p01[6 * i + 1] * 1e9, p01[6 * i + 2] * 1e9};
  const double p1[3] = {p01[6 * i + 3] * 1e9, p01[6 * i + 4] * 1e9, p01[6 * i + 5] * 1e9};
  NV r = shape_first_normal(s, shape, p0, p1);
  out[6 * i] = r.n[0];
  out[6 * i + 1] = r.n[1];
  out[6 * i + 2] = r.n[2];
  out[6 * i + 3] = r.u;
  out[6 * i + 4] = shape_contains(s, shape, p0) ? 1. : 0.;
  out[6 * i + 5] = shape_contains2(s, shape, p0, p1) ? 1. : 0.;
}

template <typename R> __global__ void k_eval_barrier(SceneView<R> s, int from, int to, int n, const double* in, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* q = in + 6 * i;
  double* o = out + 8 * i;
  R E = (R)(q[0] * kFromSIeV);
  R d[3];
  dir_from_angles(d, (R)q[1], (R)q[2]);
  double p[3] = {q[3] * 1e9, q[4] * 1e9, q[5] * 1e9};
  const double hn[3] = {0., 0., -1.};
  FixedRng<R> g{nullptr, 0, 0};
  const int reg = barrier_scatter(s, s.msms[s.regions[from].msm], p, d, E, from, to, hn, g);
  o[0] = (double)E * kEV;
  o[1] = d[0]; o[2] = d[1]; o[3] = d[2];
  o[4] = p[0] * 1e-9; o[5] = p[1] * 1e-9; o[6] = p[2] * 1e-9;
  o[7] = reg;
}

template <typename R> __global__ void k_eval_freepath(SceneView<R> s, int msm, int n, const double* in, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Msm& m = s.msms[msm];
  const R E = (R)(in[2 * i] * kFromSIeV);
  R total = 0;
  const R logE = mlog(E);
  for (int k = 0; k < m.nmech; ++k) total += mech_rate(s, s.mechs[m.mech0 + k], E, logE);
  double fp = 2.0 * kChamberRadiusNm;
  if (total != R(0)) {
    const R f = -mlog((R)in[2 * i + 1]) / total;
    if ((double)f < fp) fp = (double)f;
  }
  out[i] = fp * 1e-9;
}

}  // namespace cm

// ================================================================== C ABI
extern "C" {

const char* cm_last_error(void) { return g_err.c_str(); }
int cm_version(void) { return 1; }

}  // extern "C"
static void cm_library_anchor() {}  // an address inside this library, whoever calls
extern "C" {
const char* cm_data_dir(void) {
  if (const char* d = getenv("CM_DATA_DIR")) return d;
  static std::string dir;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  if (dir.empty()) {
    Dl_info info;
    std::string p = dladdr((void*)&cm_library_anchor, &info) && info.dli_fname ? info.dli_fname : "";
    const size_t k = p.rfind('/');
    dir = (k == std::string::npos ? std::string(".") : p.substr(0, k)) + "/data";
  }
  return dir.c_str();
}

int cm_context_create(int device, cm_context** out) {
  if (!out) return fail(CM_EINVAL, "out is null");
  int n = 0;
  CM_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(CM_EINVAL, "no such CUDA device");
  CM_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  CM_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(CM_ECUDA, "this build targets sm_100a (B200); device is sm_" +
                                                 std::to_string(prop.major) + std::to_string(prop.minor));
  std::unique_ptr<cm_context> c(new cm_context());
  c->device = device;
  c->nsm = prop.multiProcessorCount;
  // the flight kernel's call tree through nested NormalIntersectionShapes needs a few KB of local stack
  // (raised only once per device: changing the limit waits for the device to idle)
  size_t stack = 0;
  CM_CUDA(cudaDeviceGetLimit(&stack, cudaLimitStackSize));
  if (stack < 8192) CM_CUDA(cudaDeviceSetLimit(cudaLimitStackSize, 8192));
  CM_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CM_CUDA(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
  CM_CUDA(cudaMalloc(&c->counters, sizeof(Counters)));
  CM_CUDA(cudaMallocHost(&c->counters_host, sizeof(Counters)));
  CM_CUDA(cudaMallocHost(&c->io_host, sizeof(RunIO)));
  CM_CUDA(cudaHostAlloc(&c->cancel_host, sizeof(int), cudaHostAllocMapped));
  *c->cancel_host = 0;
  CM_CUDA(cudaHostGetDevicePointer((void**)&c->cancel_dev, c->cancel_host, 0));
  *out = c.release();
  return 0;
}

int cm_context_reset(cm_context* ctx) {
  if (!ctx) return fail(CM_EINVAL, "null context");
  cudaSetDevice(ctx->device);
  ctx->dirty();
  ctx->options = 0;
  ctx->mott.clear();
  ctx->tables.clear();
  ctx->mats.clear();
  ctx->msms.clear();
  ctx->shapes.clear();
  ctx->regions.clear();
  return 0;
}

int cm_context_destroy(cm_context* ctx) {
  if (!ctx) return 0;
  cudaSetDevice(ctx->device);
  ctx->dirty();
  ctx->rb64.release();
  ctx->rb32.release();
  cudaFree(ctx->counters);
  cudaFreeHost(ctx->counters_host);
  cudaFreeHost(ctx->io_host);
  cudaFreeHost(ctx->cancel_host);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  delete ctx;
  return 0;
}

int cm_get_tuning(cm_context* ctx, int precision, cm_tuning* out) {
  if (!ctx || !out) return fail(CM_EINVAL, "null argument");
  if (precision != CM_PREC_FP64 && precision != CM_PREC_FP32) return fail(CM_EINVAL, "bad precision");
  *out = ctx->tune[precision];
  return 0;
}

int cm_set_tuning(cm_context* ctx, int precision, const cm_tuning* t) {
  if (!ctx || !t) return fail(CM_EINVAL, "null argument");
  if (precision != CM_PREC_FP64 && precision != CM_PREC_FP32) return fail(CM_EINVAL, "bad precision");
  if (t->wave < 0 || (t->wave > 0 && (t->wave < 1024 || t->wave > (1 << 24)))) return fail(CM_EINVAL, "wave out of range");
  if (t->tail_below < 0) return fail(CM_EINVAL, "tail_below < 0");
  if (t->tail_steps < 0 || t->tail_steps > 4096) return fail(CM_EINVAL, "tail_steps out of range");
  if (t->blocks_per_sm < 0 || t->blocks_per_sm > 32) return fail(CM_EINVAL, "blocks_per_sm out of range");
  if (t->pool < 0 || t->pool > 64) return fail(CM_EINVAL, "pool out of range");
  ctx->tune[precision] = *t;
  return 0;
}

int cm_set_options(cm_context* ctx, int options) {
  if (!ctx) return fail(CM_EINVAL, "null context");
  ctx->options = options;
  ctx->dirty();
  return 0;
}

int cm_add_mott_element(cm_context* ctx, int Z, const double* spwem, const double* x1) {
  if (!ctx || Z < 1 || Z > 96 || !spwem || !x1) return fail(CM_EINVAL, "bad Mott element arguments");
  HMott m;
  m.spwem.assign(spwem, spwem + 61);
  m.x1.assign(x1, x1 + 61 * 201);
  ctx->mott[Z] = m;
  ctx->dirty();
  return 0;
}

int cm_add_table(cm_context* ctx, int dim, const int* n, const double* axes, const double* values, int* out) {
  if (!ctx || dim < 1 || dim > 3 || !n || !axes || !values || !out) return fail(CM_EINVAL, "bad table arguments");
  HTable t;
  memset(t.n, 0, sizeof(t.n));
  t.dim = dim;
  t.role = 0;
  t.range[0] = INFINITY;
  t.range[1] = -INFINITY;
  size_t total = 1, off = 0;
  for (int k = 0; k < dim; ++k) {
    if (n[k] < 4) return fail(CM_EINVAL, "table axes need at least 4 points");
    t.n[k] = n[k];
    t.x[k].assign(axes + off, axes + off + n[k]);
    off += n[k];
    total *= n[k];
    // a corrupt table is refused here (the reference throws on a table it cannot read,
    // NUTableInterpolation.cu:121): every abscissa finite, each axis strictly monotonic
    const std::vector<double>& x = t.x[k];
    const bool up = x[1] > x[0];
    for (int i = 0; i < n[k]; ++i) {
      if (!std::isfinite(x[i])) return fail(CM_EINVAL, "table axis " + std::to_string(k) + " has a non-finite value");
      if (i > 0 && (up ? !(x[i] > x[i - 1]) : !(x[i] < x[i - 1])))
        return fail(CM_EINVAL, "table axis " + std::to_string(k) + " is not strictly monotonic");
    }
    // NUTableInterpolation::ReadTable (:152-159)
    if (t.x[k][0] < t.x[k][n[k] - 1]) {
      t.domain[k][0] = t.x[k][0];
      t.domain[k][1] = t.x[k][n[k] - 1];
    } else {
      t.domain[k][1] = t.x[k][0];
      t.domain[k][0] = t.x[k][n[k] - 1];
    }
  }
  t.v.assign(values, values + total);
  for (double v : t.v)
    if (!std::isfinite(v)) return fail(CM_EINVAL, "table value not finite");
  for (double v : t.v) {  // (:169-172): if / else-if, as written
    if (v < t.range[0]) t.range[0] = v;
    else if (v > t.range[1]) t.range[1] = v;
  }
  *out = (int)ctx->tables.size();
  ctx->tables.push_back(t);
  ctx->dirty();
  return 0;
}

int cm_add_material(cm_context* ctx, int nel, const int* Z, const double* A, const double* wf, double density,
                    double workfunction, double ecb, double bandgap, int ncore, const double* core, int* out) {
  if (!ctx || nel < 0 || nel > kMaxElem || ncore < 0 || ncore > kMaxCore || !out) return fail(CM_EINVAL, "bad material");
  HMaterial m;
  for (int i = 0; i < nel; ++i) {
    m.Z.push_back(Z[i]);
    m.A.push_back(A[i]);
    m.wf.push_back(wf[i]);
  }
  // SEmaterial keeps core energies in a std::set: ascending, unique
  std::vector<double> c(core, core + ncore);
  std::sort(c.begin(), c.end());
  c.erase(std::unique(c.begin(), c.end()), c.end());
  m.core = c;
  m.density = density;
  m.workfunction = workfunction;
  m.ecb = ecb;
  m.bandgap = bandgap;
  *out = (int)ctx->mats.size();
  ctx->mats.push_back(m);
  ctx->dirty();
  return 0;
}

int cm_add_msm(cm_context* ctx, int material, int* out) {
  if (!ctx || material < 0 || material >= (int)ctx->mats.size() || !out) return fail(CM_EINVAL, "bad material handle");
  HMsm m;
  m.material = material;
  m.csd = 0;
  m.breakE = 0;
  m.minSet = false;
  m.minE = 0;
  m.classical = 1;
  m.lambda = 0;
  *out = (int)ctx->msms.size();
  ctx->msms.push_back(m);
  ctx->dirty();
  return 0;
}

static int add_mech(cm_context* ctx, int msm, const HMech& k, int* out) {
  if (!ctx || msm < 0 || msm >= (int)ctx->msms.size()) return fail(CM_EINVAL, "bad scatter model handle");
  auto& m = ctx->msms[msm];
  if ((int)m.mechs.size() >= kMaxMech) return fail(CM_EINVAL, "too many mechanisms");
  if (out) *out = (int)m.mechs.size();
  m.mechs.push_back(k);
  ctx->dirty();
  return 0;
}

int cm_msm_add_nistmott(cm_context* ctx, int msm, int method, int* out) {
  if (method < 1 || method > 3) return fail(CM_EINVAL, "NISTMottRS method must be 1, 2 or 3");
  HMech k;
  memset(&k, 0, sizeof(k));
  k.kind = MECH_NISTMOTT;
  k.method = method;
  return add_mech(ctx, msm, k, out);
}

int cm_msm_add_tabulated(cm_context* ctx, int msm, int method_se, double energy_offset, const int tables[4], int* out) {
  if (!ctx || !tables) return fail(CM_EINVAL, "null tables");
  const int roles[4] = {1, 2, 3, 4};
  const int dims[4] = {1, 2, 3, 2};
  for (int k = 0; k < 4; ++k) {
    if (k == 3 && method_se != 2 && method_se != 3) continue;
    if (tables[k] < 0 || tables[k] >= (int)ctx->tables.size()) return fail(CM_EINVAL, "bad table handle");
    HTable& t = ctx->tables[tables[k]];
    if (t.dim != dims[k]) return fail(CM_EINVAL, "table has the wrong dimension for its role");
    if (t.role && t.role != roles[k]) return fail(CM_EINVAL, "table used in two roles");
    t.role = roles[k];
  }
  HMech k;
  memset(&k, 0, sizeof(k));
  k.kind = MECH_TABULATED;
  k.method = method_se;
  k.energyOffset = energy_offset;
  for (int i = 0; i < 4; ++i) k.tables[i] = tables[i];
  return add_mech(ctx, msm, k, out);
}

int cm_msm_add_fitted(cm_context* ctx, int msm, double energy_se_gen, double break_e, int* out) {
  HMech k;
  memset(&k, 0, sizeof(k));
  k.kind = MECH_FITTED;
  k.energySEgen = energy_se_gen;
  k.breakE = break_e;
  return add_mech(ctx, msm, k, out);
}

int cm_msm_add_phonon(cm_context* ctx, int msm, double ratemult, double phonon_e, double temperature, double eps0,
                      double eps_inf, int* out) {
  HMech k;
  memset(&k, 0, sizeof(k));
  k.kind = MECH_PHONON;
  k.ratemult = ratemult;
  k.phononE = phonon_e;
  k.temperature = temperature;
  k.eps0 = eps0;
  k.epsInf = eps_inf;
  return add_mech(ctx, msm, k, out);
}

int cm_msm_add_polaron(cm_context* ctx, int msm, double prefactor, double extinction, int* out) {
  HMech k;
  memset(&k, 0, sizeof(k));
  k.kind = MECH_POLARON;
  k.prefactor = prefactor;
  k.extinction = extinction;
  return add_mech(ctx, msm, k, out);
}

int cm_msm_set_csd_jln(cm_context* ctx, int msm, double break_e) {
  if (!ctx || msm < 0 || msm >= (int)ctx->msms.size()) return fail(CM_EINVAL, "bad scatter model handle");
  ctx->msms[msm].csd = 1;
  ctx->msms[msm].breakE = break_e;
  ctx->dirty();
  return 0;
}

int cm_msm_set_min_e(cm_context* ctx, int msm, double min_e) {
  if (!ctx || msm < 0 || msm >= (int)ctx->msms.size()) return fail(CM_EINVAL, "bad scatter model handle");
  ctx->msms[msm].minSet = true;
  ctx->msms[msm].minE = min_e;
  ctx->dirty();
  return 0;
}

int cm_msm_set_barrier(cm_context* ctx, int msm, int classical, double lambda) {
  if (!ctx || msm < 0 || msm >= (int)ctx->msms.size()) return fail(CM_EINVAL, "bad scatter model handle");
  ctx->msms[msm].classical = classical ? 1 : 0;
  ctx->msms[msm].lambda = lambda;
  ctx->dirty();
  return 0;
}

int cm_shape_sphere(cm_context* ctx, const double center[3], double radius, int* out) {
  if (!ctx || !center || !out || !(radius > 0)) return fail(CM_EINVAL, "bad sphere");
  HShape s;
  s.kind = SHAPE_SPHERE;
  for (int k = 0; k < 3; ++k) s.c[k] = center[k];
  s.r = radius;
  s.a = s.b = -1;
  *out = (int)ctx->shapes.size();
  ctx->shapes.push_back(s);
  ctx->dirty();
  return 0;
}

int cm_shape_planes(cm_context* ctx, int n, const double* normals, const double* points, int* out) {
  if (!ctx || n < 1 || n > 64 || !normals || !points || !out) return fail(CM_EINVAL, "bad plane set");
  HShape s;
  s.kind = SHAPE_PLANES;
  s.n.assign(normals, normals + 3 * n);
  s.p.assign(points, points + 3 * n);
  s.a = s.b = -1;
  s.r = 0;
  s.c[0] = s.c[1] = s.c[2] = 0;
  *out = (int)ctx->shapes.size();
  ctx->shapes.push_back(s);
  ctx->dirty();
  return 0;
}

static int shape_depth(cm_context* ctx, int id) {
  const HShape& s = ctx->shapes[id];
  if (s.kind != SHAPE_INTERSECTION && s.kind != SHAPE_UNION) return 0;
  return 1 + std::max(shape_depth(ctx, s.a), shape_depth(ctx, s.b));
}

// NormalCylindricalShape(end0, end1, radius) (JMONSEL/NormalCylindricalShape.cu:8-17).
// Its members are initialised in declaration order (NormalCylindricalShape.cuh:29-35),
// so the reference divides the axis by a length it has not set yet (read as 0):
// the normalised axis is infinite (NaN where a component is 0) and the cylinder is
// never struck by getFirstNormal nor holds a step by contains(p0, p1).  That is
// reproduced unless CM_OPT_JMONSEL_FIXES is set when the cylinder is created.
int cm_shape_cylinder(cm_context* ctx, const double end0[3], const double end1[3], double radius, int* out) {
  if (!ctx || !end0 || !end1 || !out || !(radius > 0)) return fail(CM_EINVAL, "bad cylinder");
  HShape s;
  s.kind = SHAPE_CYLINDER;
  s.a = s.b = -1;
  s.r = 0;
  s.c[0] = s.c[1] = s.c[2] = 0;
  for (int k = 0; k < 3; ++k) {
    s.e0[k] = end0[k];
    s.ax[k] = end1[k] - end0[k];
  }
  const double len2 = (s.ax[0] * s.ax[0]) + (s.ax[1] * s.ax[1]) + (s.ax[2] * s.ax[2]);
  if (!(len2 > 0)) return fail(CM_EINVAL, "cylinder of zero length");
  s.len2 = len2;
  const double len = (ctx->options & CM_OPT_JMONSEL_FIXES) ? sqrt(len2) : 0.0;
  for (int k = 0; k < 3; ++k) s.nax[k] = s.ax[k] / len;
  s.radius = radius;
  *out = (int)ctx->shapes.size();
  ctx->shapes.push_back(s);
  ctx->dirty();
  return 0;
}

// NormalUnionShape(a, b) (JMONSEL/NormalUnionShape.cu:8-11)
int cm_shape_union(cm_context* ctx, int a, int b, int* out) {
  if (!ctx || !out || a < 0 || b < 0 || a >= (int)ctx->shapes.size() || b >= (int)ctx->shapes.size())
    return fail(CM_EINVAL, "bad shape handle");
  if (ctx->shapes[a].kind == SHAPE_SPHERE || ctx->shapes[b].kind == SHAPE_SPHERE)
    return fail(CM_EINVAL, "a Sphere is not a NormalShape");
  HShape s;
  s.kind = SHAPE_UNION;
  s.a = a;
  s.b = b;
  s.r = 0;
  s.c[0] = s.c[1] = s.c[2] = 0;
  *out = (int)ctx->shapes.size();
  ctx->shapes.push_back(s);
  if (shape_depth(ctx, *out) > kMaxShapeDepth) {
    ctx->shapes.pop_back();
    return fail(CM_EINVAL, "shape nesting deeper than 4");
  }
  ctx->dirty();
  return 0;
}

int cm_shape_intersection(cm_context* ctx, int a, int b, int* out) {
  if (!ctx || !out || a < 0 || b < 0 || a >= (int)ctx->shapes.size() || b >= (int)ctx->shapes.size())
    return fail(CM_EINVAL, "bad shape handle");
  if (ctx->shapes[a].kind == SHAPE_SPHERE || ctx->shapes[b].kind == SHAPE_SPHERE)
    return fail(CM_EINVAL, "a Sphere is not a NormalShape");
  HShape s;
  s.kind = SHAPE_INTERSECTION;
  s.a = a;
  s.b = b;
  s.r = 0;
  s.c[0] = s.c[1] = s.c[2] = 0;
  *out = (int)ctx->shapes.size();
  ctx->shapes.push_back(s);
  if (shape_depth(ctx, *out) > kMaxShapeDepth) {
    ctx->shapes.pop_back();
    return fail(CM_EINVAL, "shape nesting deeper than 4");
  }
  ctx->dirty();
  return 0;
}

static void translate_rec(cm_context* ctx, int id, const double* d) {
  HShape& s = ctx->shapes[id];
  if (s.kind == SHAPE_PLANES) {
    for (size_t i = 0; i < s.p.size(); ++i) s.p[i] += d[i % 3];  // Plane::translate (MultiPlaneShape.cu:59-64)
  } else if (s.kind == SHAPE_INTERSECTION || s.kind == SHAPE_UNION) {
    translate_rec(ctx, s.a, d);
    translate_rec(ctx, s.b, d);
  } else if (s.kind == SHAPE_CYLINDER) {
    for (int k = 0; k < 3; ++k) s.e0[k] += d[k];  // NormalCylindricalShape.cu:321-328
  } else {
    for (int k = 0; k < 3; ++k) s.c[k] += d[k];
  }
}

// Transform3D::rotation (Utility/Transform3D.cu:5-40): Euler angles phi about z, theta about y, psi about z,
// with the reference's separate form for phi == 0
static void euler_matrix(double phi, double th, double psi, double r[3][3]) {
  if (phi != 0.0) {
    const double cTh = cos(th), sTh = sin(th), cPhi = cos(phi), sPhi = sin(phi), cPsi = cos(psi), sPsi = sin(psi);
    r[0][0] = cPhi * cTh * cPsi - sPhi * sPsi;
    r[0][1] = -sPhi * cTh * cPsi - cPhi * sPsi;
    r[0][2] = sTh * cPsi;
    r[1][0] = sPhi * cPsi + cPhi * cTh * sPsi;
    r[1][1] = -sPhi * cTh * sPsi + cPhi * cPsi;
    r[1][2] = sTh * sPsi;
    r[2][0] = -cPhi * sTh;
    r[2][1] = sTh * sPhi;
    r[2][2] = cTh;
  } else {
    const double cTh = cos(th), sTh = sin(th), cPsi = cos(psi), sPsi = sin(psi);
    r[0][0] = cTh * cPsi;
    r[0][1] = -sPsi;
    r[0][2] = sTh * cPsi;
    r[1][0] = cTh * sPsi;
    r[1][1] = cPsi;
    r[1][2] = sTh * sPsi;
    r[2][0] = -sTh;
    r[2][1] = 0.0;
    r[2][2] = cTh;
  }
}

// Transform3D::rotate (Transform3D.cu:73-92, 125-128): the matrix times v, each component summed from zero
// over the columns in order; a point turns about the pivot
static void rot_vec(const double r[3][3], const double* v, double* out) {
  double o[3];
  for (int i = 0; i < 3; ++i) {
    double acc = 0.0;
    for (int k = 0; k < 3; ++k) acc += r[i][k] * v[k];
    o[i] = acc;
  }
  for (int i = 0; i < 3; ++i) out[i] = o[i];
}
static void rot_point(const double r[3][3], const double* pt, const double* pivot, double* out) {
  double d[3], q[3];
  for (int k = 0; k < 3; ++k) d[k] = pt[k] - pivot[k];
  rot_vec(r, d, q);
  for (int k = 0; k < 3; ++k) out[k] = q[k] + pivot[k];
}

static void rotate_rec(cm_context* ctx, int id, const double r[3][3], const double* pivot) {
  HShape& s = ctx->shapes[id];
  if (s.kind == SHAPE_PLANES) {  // Plane::rotate (MultiPlaneShape.cu:53-57): normal and point
    for (size_t i = 0; i + 2 < s.n.size(); i += 3) {
      rot_vec(r, &s.n[i], &s.n[i]);
      rot_point(r, &s.p[i], pivot, &s.p[i]);
    }
  } else if (s.kind == SHAPE_INTERSECTION || s.kind == SHAPE_UNION) {
    rotate_rec(ctx, s.a, r, pivot);
    rotate_rec(ctx, s.b, r, pivot);
  } else if (s.kind == SHAPE_CYLINDER) {  // NormalCylindricalShape.cu:324-330
    rot_point(r, s.e0, pivot, s.e0);
    rot_vec(r, s.ax, s.ax);
    const double l = sqrt(s.len2);
    for (int k = 0; k < 3; ++k) s.nax[k] = s.ax[k] / l;
  } else {
    rot_point(r, s.c, pivot, s.c);
  }
}

int cm_shape_rotate(cm_context* ctx, int shape, const double pivot[3], double phi, double theta, double psi) {
  if (!ctx || !pivot || shape < 0 || shape >= (int)ctx->shapes.size()) return fail(CM_EINVAL, "bad shape handle");
  double r[3][3];
  euler_matrix(phi, theta, psi, r);
  rotate_rec(ctx, shape, r, pivot);
  ctx->dirty();
  return 0;
}

int cm_shape_translate(cm_context* ctx, int shape, const double d[3]) {
  if (!ctx || !d || shape < 0 || shape >= (int)ctx->shapes.size()) return fail(CM_EINVAL, "bad shape handle");
  translate_rec(ctx, shape, d);
  ctx->dirty();
  return 0;
}

// NShapes::createLine (JMONSEL/NShapes.cu:55-149).  A corner radius turns a
// sidewall into the union of the sidewall (plus a clipping plane) and a cylinder
// along y; the reference builds the left union from the RIGHT sidewall's plane
// set (NShapes.cu:140), reproduced unless CM_OPT_JMONSEL_FIXES is set.
int cm_shape_line(cm_context* ctx, double topz, double width, double length, double thetal, double thetar,
                  double radl, double radr, int* out) {
  if (!ctx || !out) return fail(CM_EINVAL, "null argument");
  if (radr < 0.) radr = 0.;
  if (radl < 0.) radl = 0.;
  double signz = !topz ? 0 : (topz > 0 ? 1 : -1);
  if (signz == 0.) signz = 1.;
  const double en[12] = {0., 0., signz, 0., 0., -signz, 0., 1., 0., 0., -1., 0.};
  const double ep[12] = {0., 0., topz, 0., 0., 0., 0., length / 2., 0., 0., -length / 2., 0.};
  const double root2 = sqrt(2.), absz = signz * topz;
  int enclosure, rightNMPS, leftNMPS, rightSide, leftSide, nts, cyl, rc;
  if ((rc = cm_shape_planes(ctx, 4, en, ep, &enclosure))) return rc;
  const double costhetar = cos(thetar), sinthetar = sin(thetar);
  double rn[6] = {costhetar, 0., signz * sinthetar, 0, 0, 0}, rp[6] = {width / 2, 0., 0., 0, 0, 0};
  if (radr > 0) {
    const double rad = sqrt(1 - sinthetar);
    rn[3] = rad / root2;
    rn[5] = (signz * costhetar) / root2 / rad;
    rp[3] = ((width / 2.) - (radr / costhetar)) + (((radr - absz) * sinthetar) / costhetar);
    rp[5] = topz;
  }
  if ((rc = cm_shape_planes(ctx, radr > 0 ? 2 : 1, rn, rp, &rightNMPS))) return rc;
  rightSide = rightNMPS;
  if (radr > 0) {
    const double xc = ((width / 2.) - (radr / cos(thetar))) + ((radr - absz) * tan(thetar));
    const double zc = topz - (signz * radr);
    const double e0[3] = {xc, -length / 2., zc}, e1[3] = {xc, length / 2., zc};
    if ((rc = cm_shape_cylinder(ctx, e0, e1, radr, &cyl)) || (rc = cm_shape_union(ctx, rightNMPS, cyl, &rightSide)))
      return rc;
  }
  const double costhetal = cos(thetal), sinthetal = sin(thetal);
  double ln[6] = {-costhetal, 0., signz * sinthetal, 0, 0, 0}, lp[6] = {-width / 2, 0., 0., 0, 0, 0};
  if (radl > 0.) {
    const double rad = sqrt(1 - sinthetal);
    ln[3] = -rad / root2;
    ln[5] = (signz * costhetal) / root2 / rad;
    lp[3] = ((-width / 2.) + (radl / costhetal)) - (((radl - absz) * sinthetal) / costhetal);
    lp[5] = topz;
  }
  if ((rc = cm_shape_planes(ctx, radl > 0 ? 2 : 1, ln, lp, &leftNMPS))) return rc;
  leftSide = leftNMPS;
  if (radl > 0.) {
    const double xc = ((width / 2.) - (radl / cos(thetal))) + ((radl - absz) * tan(thetal));
    const double zc = topz - (signz * radl);
    const double e0[3] = {-xc, -length / 2., zc}, e1[3] = {-xc, length / 2., zc};
    const int side = (ctx->options & CM_OPT_JMONSEL_FIXES) ? leftNMPS : rightNMPS;
    if ((rc = cm_shape_cylinder(ctx, e0, e1, radl, &cyl)) || (rc = cm_shape_union(ctx, side, cyl, &leftSide))) return rc;
  }
  if ((rc = cm_shape_intersection(ctx, leftSide, rightSide, &nts))) return rc;
  return cm_shape_intersection(ctx, nts, enclosure, out);
}

int cm_region_add(cm_context* ctx, int parent, int msm, int shape, int* out) {
  if (!ctx || !out || msm < 0 || msm >= (int)ctx->msms.size() || shape < 0 || shape >= (int)ctx->shapes.size() ||
      parent >= (int)ctx->regions.size() || parent < -1)
    return fail(CM_EINVAL, "bad region arguments");
  HRegion r;
  r.parent = parent;
  r.msm = msm;
  r.shape = shape;
  *out = (int)ctx->regions.size();
  ctx->regions.push_back(r);
  if (parent >= 0) ctx->regions[parent].children.push_back(*out);
  ctx->dirty();
  return 0;
}

// ---- runs
static int check_desc(cm_context* ctx, const cm_run_desc* d) {
  if (!ctx || !d) return fail(CM_EINVAL, "null argument");
  if (d->precision != CM_PREC_FP64 && d->precision != CM_PREC_FP32) return fail(CM_EINVAL, "bad precision");
  if (d->npix < 1) return fail(CM_EINVAL, "npix < 1");
  if (d->chamber < 0 || d->chamber >= (int)ctx->regions.size()) return fail(CM_EINVAL, "bad chamber handle");
  if (ctx->regions[d->chamber].parent != -1) return fail(CM_EINVAL, "the chamber must be a root region");
  if (d->hist_stride < 3 || d->hist_stride > 1026) return fail(CM_EINVAL, "hist_stride out of range");
  if (!(d->beam_width >= 0)) return fail(CM_EINVAL, "negative beam width");
  if (d->wave < 0 || d->wave > kMaxWave) return fail(CM_EINVAL, "wave out of range (0 .. 2^27 electrons)");
  return 0;
}

struct PixelPrep {
  std::vector<double> center_nm, e0, e0ref;
  std::vector<unsigned long long> prefix, key, first;  // first: empty when the run starts every pixel at 0
  unsigned long long total = 0;
};

static int prep_pixels(const cm_run_desc* d, const double* center, const double* energy, const int* nprim,
                       const int* nbins, int stride, PixelPrep& p) {
  p.center_nm.resize(3 * (size_t)d->npix);
  p.e0.resize(d->npix);
  p.e0ref.resize(d->npix);
  p.prefix.resize(d->npix + 1);
  p.prefix[0] = 0;
  for (int i = 0; i < d->npix; ++i) {
    for (int k = 0; k < 3; ++k) {
      if (!std::isfinite(center[3 * i + k])) return fail(CM_EINVAL, "pixel centre not finite");
      p.center_nm[3 * i + k] = center[3 * i + k] * 1e9;
    }
    if (!(energy[i] > 0) || !std::isfinite(energy[i])) return fail(CM_EINVAL, "beam energy must be positive and finite");
    if (nprim[i] < 0) return fail(CM_EINVAL, "negative primary count");
    if (nbins[i] < 1 || nbins[i] + 2 > stride) return fail(CM_EINVAL, "pixel_nbins out of range");
    p.e0[i] = energy[i] * kFromSIeV;
    p.e0ref[i] = energy[i] * kFromSIeV;  // BackscatterStats: FromSI::eV(beam energy)
    p.prefix[i + 1] = p.prefix[i] + (unsigned long long)nprim[i];
  }
  p.key.resize(d->npix);
  for (int i = 0; i < d->npix; ++i)
    p.key[i] = d->pixel_key ? (unsigned long long)d->pixel_key[i]
                            : mix64(mix64(d->seed ^ 0x243F6A8885A308D3ULL) + (unsigned long long)i);
  p.total = p.prefix[d->npix];
  if (d->pixel_first) {
    p.first.resize(d->npix);
    for (int i = 0; i < d->npix; ++i) {
      if (d->pixel_first[i] < 0) return fail(CM_EINVAL, "negative pixel_first");
      p.first[i] = (unsigned long long)d->pixel_first[i];
    }
  }
  return 0;
}

extern "C++" {
template <typename T> static int up(std::vector<void*>& allocs, const std::vector<T>& v, T** out, cudaStream_t s) {
  void* ptr;
  CM_CUDA(cudaMalloc(&ptr, std::max<size_t>(1, v.size()) * sizeof(T)));
  allocs.push_back(ptr);
  CM_CUDA(cudaMemcpyAsync(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  *out = (T*)ptr;
  return 0;
}
}

static int run_common(cm_context* ctx, const cm_run_desc* d, const double* center_h, const double* energy_h,
                      const int* nprim_h, const int* nbins_h, int* nbins_dev_in, uint32_t* back_dev, uint32_t* fwd_dev,
                      cm_run_stats* st, cudaStream_t stream) {
  NvtxRange range("cm run");
  PixelPrep p;
  int rc = prep_pixels(d, center_h, energy_h, nprim_h, nbins_h, d->hist_stride, p);
  if (rc) return rc;
  std::vector<void*> allocs;
  double *c_dev, *e0_dev, *e0ref_dev;
  unsigned long long *prefix_dev, *key_dev, *first_dev = nullptr;
  int* nbins_dev = nbins_dev_in;
  std::vector<int> nb(nbins_h, nbins_h + d->npix);
  if ((rc = up(allocs, p.center_nm, &c_dev, stream)) || (rc = up(allocs, p.e0, &e0_dev, stream)) ||
      (rc = up(allocs, p.e0ref, &e0ref_dev, stream)) || (rc = up(allocs, p.prefix, &prefix_dev, stream)) ||
      (rc = up(allocs, p.key, &key_dev, stream)) ||
      (!p.first.empty() && (rc = up(allocs, p.first, &first_dev, stream))) ||
      (!nbins_dev && (rc = up(allocs, nb, &nbins_dev, stream)))) {
    for (void* a : allocs) cudaFree(a);
    return rc;
  }
  cm_run_desc dd = *d;
  dd.pixel_center = c_dev;
  dd.pixel_energy = e0_dev;
  dd.pixel_nbins = nbins_dev;
  dd.pixel_first = (const int64_t*)first_dev;  // device copy (null: every pixel from 0)
  const double emax = p.e0.empty() ? 0.0 : *std::max_element(p.e0.begin(), p.e0.end());
  NvtxRange transport("cm transport");
  rc = d->precision == CM_PREC_FP64
           ? run_device<double>(ctx, &dd, back_dev, fwd_dev, st, stream, prefix_dev, e0ref_dev, key_dev, p.total, emax)
           : run_device<float>(ctx, &dd, back_dev, fwd_dev, st, stream, prefix_dev, e0ref_dev, key_dev, p.total, emax);
  cudaStreamSynchronize(stream);
  for (void* a : allocs) cudaFree(a);
  return rc;
}

int cm_run(cm_context* ctx, const cm_run_desc* d, uint32_t* back, uint32_t* fwd, cm_run_stats* st) {
  int rc = check_desc(ctx, d);
  if (rc) return rc;
  if (!d->pixel_center || !d->pixel_energy || !d->pixel_nprim || !d->pixel_nbins || !back || !fwd)
    return fail(CM_EINVAL, "null array");
  CM_CUDA(cudaSetDevice(ctx->device));
  const size_t hbytes = (size_t)d->npix * d->hist_stride * sizeof(uint32_t);
  const bool angles = d->elevation && d->azimuth;
  const bool logged = d->escape_log && d->escape_log_cap > 0;
  const size_t ebytes = angles ? (size_t)d->npix * CM_ELEVATION_COUNTS * sizeof(uint32_t) : 0;
  const size_t abytes = angles ? (size_t)d->npix * CM_AZIMUTH_COUNTS * sizeof(uint32_t) : 0;
  const size_t lbytes = logged ? (size_t)d->escape_log_cap * sizeof(cm_escape_record) : 0;
  // device copies of the tallies: back, fwd, and when asked the angle histograms and the escape log
  std::vector<void*> bufs;
  void* dev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  const size_t sizes[5] = {hbytes, hbytes, ebytes, abytes, lbytes};
  for (int k = 0; k < 5; ++k) {
    if (!sizes[k]) continue;
    if (cudaMalloc(&dev[k], sizes[k]) != cudaSuccess) {
      (void)cudaGetLastError();
      for (void* p : bufs) cudaFree(p);
      return fail(CM_ENOMEM, "tally allocation failed");
    }
    bufs.push_back(dev[k]);
    cudaMemsetAsync(dev[k], 0, sizes[k], ctx->stream);
  }
  cm_run_desc dl = *d;
  dl.elevation = (uint32_t*)dev[2];
  dl.azimuth = (uint32_t*)dev[3];
  dl.escape_log = (cm_escape_record*)dev[4];
  rc = run_common(ctx, &dl, d->pixel_center, d->pixel_energy, d->pixel_nprim, d->pixel_nbins, nullptr, (uint32_t*)dev[0],
                  (uint32_t*)dev[1], st, ctx->stream);
  if (!rc) {
    cudaMemcpyAsync(back, dev[0], hbytes, cudaMemcpyDeviceToHost, ctx->stream);
    cudaMemcpyAsync(fwd, dev[1], hbytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (angles) {
      cudaMemcpyAsync(d->elevation, dev[2], ebytes, cudaMemcpyDeviceToHost, ctx->stream);
      cudaMemcpyAsync(d->azimuth, dev[3], abytes, cudaMemcpyDeviceToHost, ctx->stream);
    }
    if (logged && st) {
      const int64_t n = std::min<int64_t>(d->escape_log_cap, st->escapes);
      cudaMemcpyAsync(d->escape_log, dev[4], (size_t)n * sizeof(cm_escape_record), cudaMemcpyDeviceToHost, ctx->stream);
    } else if (logged) {
      cudaMemcpyAsync(d->escape_log, dev[4], lbytes, cudaMemcpyDeviceToHost, ctx->stream);
    }
    cudaStreamSynchronize(ctx->stream);
  }
  for (void* p : bufs) cudaFree(p);
  if (!rc) CM_CUDA(cudaGetLastError());
  return rc;
}

int cm_run_device(cm_context* ctx, const cm_run_desc* d, uint32_t* back, uint32_t* fwd, cm_run_stats* st, void* stream) {
  int rc = check_desc(ctx, d);
  if (rc) return rc;
  if (!d->pixel_center || !d->pixel_energy || !d->pixel_nprim || !d->pixel_nbins || !back || !fwd)
    return fail(CM_EINVAL, "null array");
  CM_CUDA(cudaSetDevice(ctx->device));
  // the loop is captured into a graph on the engine's own stream; the caller's
  // stream (possibly the legacy default stream, which cannot be captured) is
  // ordered before and after it with events
  cudaStream_t caller = (cudaStream_t)stream;
  cudaStream_t s = ctx->stream;
  cudaEvent_t ein, eout;
  CM_CUDA(cudaEventCreateWithFlags(&ein, cudaEventDisableTiming));
  CM_CUDA(cudaEventCreateWithFlags(&eout, cudaEventDisableTiming));
  CM_CUDA(cudaEventRecord(ein, caller));
  CM_CUDA(cudaStreamWaitEvent(s, ein, 0));
  // the small per-pixel arrays are read back to build the primary prefix and the unit conversions
  std::vector<double> c(3 * (size_t)d->npix), e(d->npix);
  std::vector<int> np(d->npix), nb(d->npix);
  CM_CUDA(cudaMemcpyAsync(c.data(), d->pixel_center, c.size() * 8, cudaMemcpyDeviceToHost, s));
  CM_CUDA(cudaMemcpyAsync(e.data(), d->pixel_energy, e.size() * 8, cudaMemcpyDeviceToHost, s));
  CM_CUDA(cudaMemcpyAsync(np.data(), d->pixel_nprim, np.size() * 4, cudaMemcpyDeviceToHost, s));
  CM_CUDA(cudaMemcpyAsync(nb.data(), d->pixel_nbins, nb.size() * 4, cudaMemcpyDeviceToHost, s));
  std::vector<uint64_t> keys;
  std::vector<int64_t> firsts;
  cm_run_desc dh = *d;
  if (d->pixel_key) {
    keys.resize(d->npix);
    CM_CUDA(cudaMemcpyAsync(keys.data(), d->pixel_key, keys.size() * 8, cudaMemcpyDeviceToHost, s));
    dh.pixel_key = keys.data();
  }
  if (d->pixel_first) {
    firsts.resize(d->npix);
    CM_CUDA(cudaMemcpyAsync(firsts.data(), d->pixel_first, firsts.size() * 8, cudaMemcpyDeviceToHost, s));
    dh.pixel_first = firsts.data();
  }
  CM_CUDA(cudaStreamSynchronize(s));
  d = &dh;
  const size_t hbytes = (size_t)d->npix * d->hist_stride * sizeof(uint32_t);
  CM_CUDA(cudaMemsetAsync(back, 0, hbytes, s));
  CM_CUDA(cudaMemsetAsync(fwd, 0, hbytes, s));
  if ((rc = clear_angles(d, s))) return rc;
  rc = run_common(ctx, d, c.data(), e.data(), np.data(), nb.data(), (int*)d->pixel_nbins, back, fwd, st, s);
  cudaEventRecord(eout, s);
  cudaStreamWaitEvent(caller, eout, 0);
  cudaEventDestroy(ein);
  cudaEventDestroy(eout);
  return rc;
}

// Coordinate descent over the launch settings from the defaults, one cm_run per candidate.
int cm_autotune(cm_context* ctx, const cm_run_desc* d, cm_tuning* best) {
  int rc = check_desc(ctx, d);
  if (rc) return rc;
  if (!d->pixel_center || !d->pixel_energy || !d->pixel_nprim || !d->pixel_nbins) return fail(CM_EINVAL, "null array");
  cm_run_desc dd = *d;
  dd.wave = 0;
  dd.profile = 0;
  dd.elevation = dd.azimuth = nullptr;
  dd.escape_log = nullptr;
  dd.escape_log_cap = 0;
  std::vector<uint32_t> back((size_t)d->npix * d->hist_stride), fwd(back.size());
  cm_tuning& slot = ctx->tune[d->precision];
  const cm_tuning saved = slot;
  auto trial = [&](const cm_tuning& t, double& ms) -> int {
    NvtxRange range("cm autotune trial");
    slot = t;
    cm_run_stats st;
    memset(&st, 0, sizeof(st));
    const int r = cm_run(ctx, &dd, back.data(), fwd.data(), &st);
    ms = st.device_ms;
    return r;
  };
  cm_tuning cur = d->precision == CM_PREC_FP64 ? cm::resolved_tuning<double>(ctx) : cm::resolved_tuning<float>(ctx);
  double cur_ms = 0, ms = 0;
  if ((rc = trial(cur, cur_ms)) || (rc = trial(cur, cur_ms))) {  // the first run also builds the scene
    slot = saved;
    return rc;
  }
  const int belows[] = {65536, 131072, 524288};
  const int steps[] = {16, 64};
  auto sweep = [&](int cm_tuning::*field, const int* vals, int n) -> int {
    for (int k = 0; k < n; ++k) {
      if (vals[k] == cur.*field) continue;
      cm_tuning t = cur;
      t.*field = vals[k];
      const int r = trial(t, ms);
      if (r == CM_ENOMEM) continue;  // a candidate wave that does not fit is skipped
      if (r) return r;
      if (ms < 0.99 * cur_ms) {
        cur = t;
        cur_ms = ms;
      }
    }
    return 0;
  };
  // passes of coordinate descent until one changes nothing (at most 3): the wave and the blocks per SM are
  // tried at half and twice their current values, so a later pass can go on in the direction that paid
  for (int pass = 0; pass < 3; ++pass) {
    const cm_tuning before = cur;
    const int waves[] = {std::max(1024, cur.wave / 2), std::min(1 << 24, cur.wave * 2)};
    const int blocks[] = {std::max(2, cur.blocks_per_sm / 2), std::min(32, cur.blocks_per_sm * 2)};
    if ((rc = sweep(&cm_tuning::wave, waves, 2)) || (rc = sweep(&cm_tuning::tail_below, belows, 3)) ||
        (rc = sweep(&cm_tuning::tail_steps, steps, 2)) || (rc = sweep(&cm_tuning::blocks_per_sm, blocks, 2))) {
      slot = saved;
      return rc;
    }
    if (cur.wave == before.wave && cur.tail_below == before.tail_below && cur.tail_steps == before.tail_steps &&
        cur.blocks_per_sm == before.blocks_per_sm)
      break;
  }
  cur.ms = cur_ms;
  slot = cur;
  if (best) *best = cur;
  return 0;
}

// ---- per-function entry points
extern "C++" {
template <typename F>
static int eval_launch(cm_context* ctx, int n, const double* in, size_t in_per, double* out, size_t out_per, F launch) {
  if (n < 0) return fail(CM_EINVAL, "n < 0");
  if (n == 0) return 0;
  CM_CUDA(cudaSetDevice(ctx->device));
  double *din = nullptr, *dout = nullptr;
  CM_CUDA(cudaMalloc(&din, std::max<size_t>(1, n * in_per) * 8));
  if (cudaMalloc(&dout, n * out_per * 8) != cudaSuccess) {
    cudaFree(din);
    return fail(CM_ENOMEM, "eval allocation failed");
  }
  if (in_per) cudaMemcpy(din, in, n * in_per * 8, cudaMemcpyHostToDevice);
  launch(din, dout, (n + 127) / 128);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, n * out_per * 8, cudaMemcpyDeviceToHost);
  cudaFree(din);
  cudaFree(dout);
  if (e != cudaSuccess) return fail(CM_ECUDA, cudaGetErrorString(e));
  CM_CUDA(cudaGetLastError());
  return 0;
}

}

static int scene_for(cm_context* ctx, int precision) {
  if (!ctx) return fail(CM_EINVAL, "null context");
  CM_CUDA(cudaSetDevice(ctx->device));
  if (precision == CM_PREC_FP64) return build_scene<double>(ctx, ctx->d64);
  if (precision == CM_PREC_FP32) return build_scene<float>(ctx, ctx->d32);
  return fail(CM_EINVAL, "bad precision");
}

static int mech_index(cm_context* ctx, int msm, int mech, int kind) {
  if (msm < 0 || msm >= (int)ctx->msms.size()) return -1;
  if (mech < 0 || mech >= (int)ctx->msms[msm].mechs.size()) return -1;
  if (kind && ctx->msms[msm].mechs[mech].kind != kind) return -1;
  int base = 0;
  for (int i = 0; i < msm; ++i) base += (int)ctx->msms[i].mechs.size();
  return base + mech;
}

int cm_eval_nistmott(cm_context* ctx, int Z, int method, int n, const double* E, const double* u, double* sigma,
                     double* theta, int precision) {
  if (method < 1 || method > 3) return fail(CM_EINVAL, "NISTMottRS method must be 1, 2 or 3");
  int rc = scene_for(ctx, precision);
  if (rc) return rc;
  auto it = ctx->mott.find(Z);
  if (it == ctx->mott.end()) return fail(CM_EINVAL, "element not loaded");
  const int mi = (int)std::distance(ctx->mott.begin(), it);
  std::vector<double> in(3 * (size_t)n), out(2 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    in[i] = E[i];
    in[n + 2 * i] = u[2 * i];
    in[n + 2 * i + 1] = u[2 * i + 1];
  }
  rc = eval_launch(ctx, 1, in.data(), 3 * (size_t)n, out.data(), 2 * (size_t)n, [&](double* din, double* dout, int) {
    const int g = (n + 127) / 128;
    if (precision == CM_PREC_FP64)
      k_eval_nistmott<double><<<g, 128>>>(ctx->d64.view, mi, method, n, din, din + n, dout, dout + n);
    else
      k_eval_nistmott<float><<<g, 128>>>(ctx->d32.view, mi, method, n, din, din + n, dout, dout + n);
  });
  if (rc) return rc;
  for (int i = 0; i < n; ++i) {
    sigma[i] = out[i];
    theta[i] = out[n + i];
  }
  return 0;
}

int cm_eval_table(cm_context* ctx, int table, int n, const double* x, int order, double* out, int precision) {
  int rc = scene_for(ctx, precision);
  if (rc) return rc;
  if (table < 0 || table >= (int)ctx->tables.size()) return fail(CM_EINVAL, "bad table handle");
  const HTable& t = ctx->tables[table];
  const double f0 = t.role >= 1 ? kFromSIeV : 1.0;
  const double vf = t.role == 1 ? 1e-9 : t.role == 4 ? kFromSIeV : 1.0;
  return eval_launch(ctx, n, x, 3, out, 1, [&](double* din, double* dout, int g) {
    if (precision == CM_PREC_FP64)
      k_eval_table<double><<<g, 128>>>(ctx->d64.view, table, n, din, f0, vf, order, dout);
    else
      k_eval_table<float><<<g, 128>>>(ctx->d32.view, table, n, din, f0, vf, order, dout);
  });
}

int cm_eval_locate(cm_context* ctx, int table, int n, const double* x, int order, int* out, int precision) {
  int rc = scene_for(ctx, precision);
  if (rc) return rc;
  if (table < 0 || table >= (int)ctx->tables.size()) return fail(CM_EINVAL, "bad table handle");
  if (!out) return fail(CM_EINVAL, "null output");
  const double f0 = ctx->tables[table].role >= 1 ? kFromSIeV : 1.0;
  std::vector<double> w((size_t)std::max(n, 0) * 6);
  rc = eval_launch(ctx, n, x, 3, w.data(), 6, [&](double* din, double* dout, int g) {
    if (precision == CM_PREC_FP64) k_eval_locate<double><<<g, 128>>>(ctx->d64.view, table, n, din, f0, order, dout);
    else k_eval_locate<float><<<g, 128>>>(ctx->d32.view, table, n, din, f0, order, dout);
  });
  if (rc) return rc;
  for (size_t k = 0; k < w.size(); ++k) out[k] = (int)w[k];
  return 0;
}

int cm_eval_pick(cm_context* ctx, int msm, int n, const double* in, double* out, int precision) {
  int rc = scene_for(ctx, precision);
  if (rc) return rc;
  if (msm < 0 || msm >= (int)ctx->msms.size()) return fail(CM_EINVAL, "bad material model handle");
  return eval_launch(ctx, n, in, 2, out, 2, [&](double* din, double* dout, int g) {
    if (precision == CM_PREC_FP64) k_eval_pick<double><<<g, 128>>>(ctx->d64.view, msm, n, din, dout);
    else k_eval_pick<float><<<g, 128>>>(ctx->d32.view, msm, n, din, dout);
  });
}

int cm_eval_tabulated(cm_context* ctx, int msm, int mech, int n, const double* in, double* out, int precision) {
  int rc = scene_for(ctx, precision);
  if (rc) return rc;
  const int k = mech_index(ctx, msm, mech, MECH_TABULATED);
  if (k < 0) return fail(CM_EINVAL, "not a TabulatedInelasticSM");
  return eval_launch(ctx, n, in, 9, out, 12, [&](double* din, double* dout, int g) {
    if (precision == CM_PREC_FP64) k_eval_tabulated<double><<<g, 128>>>(ctx->d64.view, k, n, din, dout);
    else k_eval_tabulated<float><<<g, 128>>>(ctx->d32.view, k, n, din, dout);
  });
}

int cm_eval_elastic(cm_context* ctx, int msm, int mech, int n, const double* in, double* out, int precision) {
  int rc = scene_for(ctx, precision);
  if (rc) return rc;
  const int k = mech_index(ctx, msm, mech, MECH_NISTMOTT);
  if (k < 0) return fail(CM_EINVAL, "not a SelectableElasticSM");
  return eval_launch(ctx, n, in, 7, out, 6, [&](double* din, double* dout, int g) {
    if (precision == CM_PREC_FP64) k_eval_elastic<double><<<g, 128>>>(ctx->d64.view, k, n, din, dout);
    else k_eval_elastic<float><<<g, 128>>>(ctx->d32.view, k, n, din, dout);
  });
}

int cm_eval_csd(cm_context* ctx, int msm, int n, const double* in, double* out, int precision) {
  int rc = scene_for(ctx, precision);
  if (rc) return rc;
  if (msm < 0 || msm >= (int)ctx->msms.size()) return fail(CM_EINVAL, "bad scatter model handle");
  return eval_launch(ctx, n, in, 2, out, 3, [&](double* din, double* dout, int g) {
    if (precision == CM_PREC_FP64) k_eval_csd<double><<<g, 128>>>(ctx->d64.view, msm, n, din, dout);
    else k_eval_csd<float><<<g, 128>>>(ctx->d32.view, msm, n, din, dout);
  });
}

int cm_eval_phonon(cm_context* ctx, int msm, int mech, int n, const double* in, double* out, int precision) {
  int rc = scene_for(ctx, precision);
  if (rc) return rc;
  const int k = mech_index(ctx, msm, mech, MECH_PHONON);
  if (k < 0) return fail(CM_EINVAL, "not a GanachaudMokraniPhononInelasticSM");
  return eval_launch(ctx, n, in, 5, out, 6, [&](double* din, double* dout, int g) {
    if (precision == CM_PREC_FP64) k_eval_phonon<double><<<g, 128>>>(ctx->d64.view, k, n, din, dout);
    else k_eval_phonon<float><<<g, 128>>>(ctx->d32.view, k, n, din, dout);
  });
}

int cm_eval_shape(cm_context* ctx, int shape, int n, const double* p01, double* out) {
  int rc = scene_for(ctx, CM_PREC_FP64);
  if (rc) return rc;
  if (shape < 0 || shape >= (int)ctx->shapes.size()) return fail(CM_EINVAL, "bad shape handle");
  return eval_launch(ctx, n, p01, 6, out, 6, [&](double* din, double* dout, int g) {
    k_eval_shape<<<g, 128>>>(ctx->d64.view, shape, n, din, dout);
  });
}

int cm_eval_barrier(cm_context* ctx, int from, int to, int n, const double* in, double* out, int precision) {
  int rc = scene_for(ctx, precision);
  if (rc) return rc;
  if (from < 0 || to < 0 || from >= (int)ctx->regions.size() || to >= (int)ctx->regions.size())
    return fail(CM_EINVAL, "bad region handle");
  return eval_launch(ctx, n, in, 6, out, 8, [&](double* din, double* dout, int g) {
    if (precision == CM_PREC_FP64) k_eval_barrier<double><<<g, 128>>>(ctx->d64.view, from, to, n, din, dout);
    else k_eval_barrier<float><<<g, 128>>>(ctx->d32.view, from, to, n, din, dout);
  });
}

int cm_eval_freepath(cm_context* ctx, int msm, int n, const double* in, double* out, int precision) {
  int rc = scene_for(ctx, precision);
  if (rc) return rc;
  if (msm < 0 || msm >= (int)ctx->msms.size()) return fail(CM_EINVAL, "bad scatter model handle");
  return eval_launch(ctx, n, in, 2, out, 1, [&](double* din, double* dout, int g) {
    if (precision == CM_PREC_FP64) k_eval_freepath<double><<<g, 128>>>(ctx->d64.view, msm, n, din, dout);
    else k_eval_freepath<float><<<g, 128>>>(ctx->d32.view, msm, n, din, dout);
  });
}

}  // extern "C"

// ================================================================== allocation-free run
// cm_run_noalloc: the transport run of cm_run_device for callers that cannot
// allocate device memory when they run trajectories -- a service whose device
// memory is owned and budgeted by another allocator (a caching pool, a fixed
// reservation made at start-up), where a cudaMalloc would be refused, would
// break that allocator's accounting or would stall the device.  Its scratch
// (wave records, secondary pool, event queues, counters, per-pixel tables)
// lives in one file-scope device array of fixed size, reserved on every GPU
// that loads the library for as long as the process lives.  The caller passes
// the pixel inputs and the tally outputs, as for cm_run_device.
namespace cm {

constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;  // 32 MiB
constexpr int kNoAllocMaxPix = 65536;
constexpr int kNoAllocMaxDevices = 64;
constexpr double kFromSIeVc = 1.0 / 1.60217653e-19;  // FromSI::EV, as kFromSIeV

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[kNoAllocMaxDevices];  // device address of g_noalloc_scratch, per device

// The per-pixel tables prep_pixels builds on the host, built here on the
// device from the caller's device arrays: centres in nm, energies in eV, the
// exclusive prefix of primaries per pixel and the per-pixel stream keys.  One
// block of 1024 threads.  A bad input sets *bad instead of running.
__global__ void k_noalloc_pixels(int n, int stride, const double* center_m, const double* energy_j, const int* nprim,
                                 const int* nbins, const uint64_t* keys, unsigned long long seedmix, double* pc,
                                 double* pe0, unsigned long long* pkey, unsigned long long* prefix, Counters* c,
                                 int* bad, RunIO* io, double width_nm, uint32_t* back, uint32_t* fwd) {
  __shared__ unsigned long long part[1024];
  if (threadIdx.x == 0) {  // the run's inputs and tallies as the transport kernels read them
    memset(io, 0, sizeof(RunIO));
    io->pc = pc;
    io->pe0 = pe0;
    io->pe0ref = pe0;  // BackscatterStats: FromSI::eV(beam energy), the same value
    io->pnbins = nbins;
    io->prefix = prefix;
    io->pkey = pkey;
    io->npix = n;
    io->width = width_nm;
    io->back = back;
    io->fwd = fwd;
    io->stride = stride;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    for (int k = 0; k < 3; ++k) pc[3 * i + k] = center_m[3 * i + k] * 1e9;
    pe0[i] = energy_j[i] * kFromSIeVc;
    pkey[i] = keys ? (unsigned long long)keys[i] : mix64(seedmix + (unsigned long long)i);
    if (!(energy_j[i] > 0) || nprim[i] < 0 || nbins[i] < 1 || nbins[i] + 2 > stride) atomicExch(bad, 1);
  }
  const int chunk = (n + (int)blockDim.x - 1) / (int)blockDim.x;
  const int lo = (int)threadIdx.x * chunk, hi = min(n, lo + chunk);
  unsigned long long sum = 0;
  for (int i = lo; i < hi; ++i) sum += (unsigned long long)max(nprim[i], 0);
  part[threadIdx.x] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long acc = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      const unsigned long long x = part[t];
      part[t] = acc;
      acc += x;
    }
    prefix[n] = acc;
    c->total_primaries = acc;
  }
  __syncthreads();
  unsigned long long acc = part[threadIdx.x];
  for (int i = lo; i < hi; ++i) {
    prefix[i] = acc;
    acc += (unsigned long long)max(nprim[i], 0);
  }
}

// bump allocator over the scratch array; every piece starts on a 256-byte boundary
struct Carve {
  unsigned char* base;
  size_t off = 0;
  template <typename T> T* take(size_t count) {
    T* p = (T*)(base + off);
    off += (count * sizeof(T) + 255) & ~(size_t)255;
    return p;
  }
};

template <typename R> static void carve_wave(Carve& a, Wave<R>& w, int cap) {
  w.px = a.take<double>(cap);
  w.py = a.take<double>(cap);
  w.pz = a.take<double>(cap);
  w.dx = a.take<R>(cap);
  w.dy = a.take<R>(cap);
  w.dz = a.take<R>(cap);
  w.E = a.take<R>(cap);
  w.Ep = a.take<R>(cap);
  w.region = a.take<int>(cap);
  w.pixel = a.take<int>(cap);
  w.aux = a.take<int>(cap);
  w.step = a.take<uint32_t>(cap);
  w.key = a.take<unsigned long long>(cap);
  w.hx = a.take<R>(cap);
  w.hy = a.take<R>(cap);
  w.hz = a.take<R>(cap);
}

template <typename R>
static int run_noalloc(cm_context* ctx, const cm_run_desc* d, uint32_t* back, uint32_t* fwd, cm_run_stats* st,
                       cudaStream_t s, unsigned char* scratch) {
  DevScene<R>& ds = scene_of<R>(ctx);
  if (!ds.valid || ds.host)
    return fail(CM_ESTATE, "cm_run_noalloc: the scene is not on the device for this precision; uploading it "
                           "allocates, so make one cm_run, cm_run_device or cm_eval_* call with this precision "
                           "after the last scene change first");
  const int n = d->npix;
  // layout: counters | bad flag | run inputs | pixel tables | wave 0 | wave 1 (kSegments W each) | 3 queues |
  // pool (8 W)
  Carve a{scratch};
  Counters* c = a.take<Counters>(1);
  int* bad = a.take<int>(1);
  RunIO* io = a.take<RunIO>(1);
  double* pc = a.take<double>(3 * (size_t)n);
  double* pe0 = a.take<double>(n);
  unsigned long long* pkey = a.take<unsigned long long>(n);
  unsigned long long* prefix = a.take<unsigned long long>((size_t)n + 1);
  // bytes per electron record: position (3 double), direction, pre-step
  // direction (3 R each), E and Ep (R), region, pixel, aux, step (4 B each), key (8 B)
  const size_t rec = 3 * 8 + 8 * sizeof(R) + 4 * 4 + 8;
  const size_t pad = (3 * 16 + 3) * 256;  // worst-case rounding of the 51 pieces below
  const size_t left = kNoAllocScratchBytes - a.off;
  long long W = (long long)((left > pad ? left - pad : 0) / ((2 * kSegments + 8) * rec + 3 * 4));
  if (d->wave > 0 && d->wave < W) W = d->wave;
  if (W < 1024) return fail(CM_EINVAL, "cm_run_noalloc: no room for a wave of 1024 electrons");
  const int poolCap = (int)(8 * W);
  RunView<R> v;
#ifdef CM_TRACE
  v.trace = nullptr;
  v.ntrace = nullptr;
  v.tracecap = 0;
#endif
  v.s = ds.view;
  v.s.chamber = d->chamber;
  carve_wave(a, v.w[0], kSegments * (int)W);
  carve_wave(a, v.w[1], kSegments * (int)W);
  for (int k = 0; k < 3; ++k) v.q[k] = a.take<int>(W);
  carve_wave(a, v.pool, poolCap);
  if (a.off > kNoAllocScratchBytes) return fail(CM_EINVAL, "cm_run_noalloc: scratch layout does not fit");
  v.c = c;
  v.W = (int)W;
  v.poolCap = poolCap;
  v.io = io;  // written by k_noalloc_pixels (no angle histograms or escape log: no room in the fixed scratch)
  // the array keeps the previous call's contents: the counters, the bad-input
  // flag and the caller's tallies start at zero; waves, queues and pool are
  // only read below the counts, so they need no clearing
  const size_t hbytes = (size_t)n * d->hist_stride * sizeof(uint32_t);
  CM_CUDA(cudaMemsetAsync(c, 0, sizeof(Counters), s));
  CM_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
  CM_CUDA(cudaMemsetAsync(back, 0, hbytes, s));
  CM_CUDA(cudaMemsetAsync(fwd, 0, hbytes, s));
  k_noalloc_pixels<<<1, 1024, 0, s>>>(n, d->hist_stride, d->pixel_center, d->pixel_energy, d->pixel_nprim,
                                      d->pixel_nbins, d->pixel_key, mix64(d->seed ^ 0x243F6A8885A308D3ULL), pc, pe0,
                                      pkey, prefix, c, bad, io, d->beam_width * 1e9, back, fwd);
  CM_CUDA(cudaGetLastError());
  int hbad = 0;
  CM_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  CM_CUDA(cudaStreamSynchronize(s));
  if (hbad)
    return fail(CM_EINVAL, "cm_run_noalloc: a pixel has a non-positive energy, a negative primary count or "
                           "pixel_nbins out of range");
  const int grid = ctx->nsm * 8;
  const int maxIt = d->max_iterations > 0 ? d->max_iterations : 500000;
  Counters hc;
  memset(&hc, 0, sizeof(hc));
  const auto t0 = std::chrono::steady_clock::now();
  int it = 0, status = 0;
  for (;;) {
    for (int k = 0; k < 16; ++k, ++it) {
      const int cur = it & 1;
      launch_flight(v, cur, grid, s);
      k_elastic<R><<<grid, 256, 0, s>>>(v, cur);
      k_inelastic<R><<<grid, 256, 0, s>>>(v, cur);
      launch_misc<R>(v, cur, grid, s);
      launch_spawn<R>(v, cur, grid, s);
      k_tail<R><<<1, 32, 0, s>>>(v, cur, 0);
    }
    CM_CUDA(cudaGetLastError());
    CM_CUDA(cudaMemcpyAsync(&hc, c, sizeof(Counters), cudaMemcpyDeviceToHost, s));
    CM_CUDA(cudaStreamSynchronize(s));
    if (hc.error) {
      status = hc.error == CM_EOVERFLOW
                   ? fail(CM_EOVERFLOW, "cm_run_noalloc: the secondary pool in the fixed scratch overflowed; pass "
                                        "fewer primaries per call or use cm_run_device")
                   : fail(hc.error, "cm_run_noalloc: the transport kernels reported error " + std::to_string(hc.error));
      break;
    }
    if (hc.done) break;
    if (ctx->cancel && ctx->cancel->load()) {
      status = fail(CM_ECANCELED, "cancelled");
      break;
    }
    if (it >= maxIt) {
      status = fail(CM_ELIMIT, "cm_run_noalloc: iteration limit reached");
      break;
    }
  }
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (st) {
    memset(st, 0, sizeof(*st));
    st->primaries = (int64_t)hc.next_primary;
    st->steps = (int64_t)hc.steps;
    st->scatter_events = (int64_t)hc.scatters;
    st->barrier_events = (int64_t)hc.barriers;
    st->escapes = (int64_t)hc.escapes;
    st->secondaries = (int64_t)hc.secondaries;
    st->iterations = (int64_t)hc.iterations;
    st->device_ms = ms;
    st->ended_zero_energy = (int64_t)hc.ended_zero;
    st->ended_step_limit = (int64_t)hc.ended_limit;
    for (int k = 0; k < 6; ++k) st->kernel_launches[k] = it;
    for (int k = 0; k < 4; ++k) st->units[k] = (int64_t)hc.units[k];
  }
  return status;
}

}  // namespace cm

extern "C" int cm_run_noalloc(cm_context* ctx, const cm_run_desc* d, uint32_t* back, uint32_t* fwd,
                              cm_run_stats* stats, void* stream) {
  using namespace cm;
  int rc = check_desc(ctx, d);
  if (!rc && (d->elevation || d->azimuth || d->escape_log))
    rc = fail(CM_EINVAL, "cm_run_noalloc tallies the energy histograms only (no angle histograms or escape log)");
  if (!rc && d->pixel_first) rc = fail(CM_EINVAL, "cm_run_noalloc starts every pixel at its primary 0 (no pixel_first)");
  if (rc) return rc;
  if (!d->pixel_center || !d->pixel_energy || !d->pixel_nprim || !d->pixel_nbins || !back || !fwd)
    return fail(CM_EINVAL, "null array");
  if (d->npix > kNoAllocMaxPix)
    return fail(CM_EINVAL, "cm_run_noalloc: npix " + std::to_string(d->npix) + " exceeds its maximum of " +
                               std::to_string(kNoAllocMaxPix));
  if (ctx->device < 0 || ctx->device >= kNoAllocMaxDevices)
    return fail(CM_EINVAL, "cm_run_noalloc: device index beyond " + std::to_string(kNoAllocMaxDevices));
  CM_CUDA(cudaSetDevice(ctx->device));
  void* scratch;
  {
    // set-up on the first call on each device, with that device current: the
    // host-side name of the array is only a stand-in, the runtime gives its
    // device address
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[ctx->device]) {
      void* ptr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr)
        return fail(CM_ECUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
      g_noalloc_addr[ctx->device] = ptr;
    }
    scratch = g_noalloc_addr[ctx->device];
  }
  cudaStream_t s = (cudaStream_t)stream;
  return d->precision == CM_PREC_FP64 ? run_noalloc<double>(ctx, d, back, fwd, stats, s, (unsigned char*)scratch)
                                      : run_noalloc<float>(ctx, d, back, fwd, stats, s, (unsigned char*)scratch);
}

#include "cm_server.cuh"
