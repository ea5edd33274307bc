/*
 * cudamonsel_b200.hpp -- the reference's C++ API for the transport path, over the C ABI of
 * cudamonsel_b200.h.  A driver written against CudaMONSEL's classes (JMONSELTests/LinesOnLayers.cu:80-388:
 * SEmaterial, the ScatterMechanism / SlowingDownAlg / BarrierScatterMechanism plug-ins,
 * MONSEL_MaterialScatterModel, the Normal shapes and NShapes::createLine, Region, GaussianBeam,
 * MonteCarloSS and BackscatterStats) compiles against this header unchanged and runs its trajectories on
 * the GPU.  Link with -lcudamonsel_b200.
 *
 * The objects record what the driver builds; the first MonteCarloSS::runMultipleTrajectories after a change
 * replays the Region tree under the chamber into an engine context (materials, mechanisms and tables
 * once each, shapes with the translations and rotations applied to them so far) and every run tallies into
 * the BackscatterStats listening to it.  Differences from the reference, all documented here:
 *   - errors throw cudamonsel::Error (the reference prints and carries on, or throws 0);
 *   - random numbers are the engine's counter-based streams: run k of a process uses seed
 *     cudamonsel::seed() + k (cudamonsel::set_seed), so results are reproducible run by run;
 *   - transport runs in FP32 with FP64 positions and plane solves unless cudamonsel::set_precision
 *     selects CM_PREC_FP64 (the reference is all FP64);
 *   - ActionListeners other than BackscatterStats are not called (the GPU has no per-event callbacks);
 *   - a shape changed after a run has used it is replayed on the next run (the reference reads it live);
 *   - translating or rotating an intersection or union moves its parts (the reference's casts there are
 *     unsafe to run), and a rotation also normalises the axis of a cylinder, as in the reference;
 *   - cudamonsel::set_options(CM_OPT_*) selects the engine options: cylinders and rounded lines take
 *     those set when they are constructed, everything else those set when a run starts.
 * NIST Mott data are read from the library's data directory ($CM_DATA_DIR, else the "data" folder beside
 * libcudamonsel_b200.so); scattering tables from the paths the driver names.
 */
#ifndef CUDAMONSEL_B200_HPP
#define CUDAMONSEL_B200_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cudamonsel_b200.h"

typedef std::string StringT;
typedef std::vector<double> VectorXd;

namespace cudamonsel {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const char* what) {
  if (rc != 0) throw Error(rc, std::string(what) + ": " + cm_last_error());
}

// the process's engine context and settings (the reference's objects are process-wide too)
struct Session {
  cm_context* ctx = nullptr;
  int precision = CM_PREC_FP32;
  int options = 0;
  uint64_t seed = 0;
  uint64_t runs = 0;
  unsigned long long version = 1;  // bumped by every change to a recorded object
  // the settings, without touching the GPU
  static Session& state() {
    static Session s;
    return s;
  }
  // the settings and the engine context ($CM_DEVICE, else device 0), created on first use
  static Session& get() {
    Session& s = state();
    if (!s.ctx) {
      const char* dev = getenv("CM_DEVICE");
      check(cm_context_create(dev ? atoi(dev) : 0, &s.ctx), "cm_context_create");
    }
    return s;
  }
  ~Session() {
    if (ctx) cm_context_destroy(ctx);
  }
};
inline void touch() { Session::state().version++; }
inline void set_precision(int precision) { Session::state().precision = precision; }
inline void set_options(int options) { Session::state().options = options; touch(); }
inline void set_seed(uint64_t s) { Session::state().seed = s; Session::state().runs = 0; }
inline uint64_t seed() { return Session::state().seed; }
inline cm_context* context() { return Session::get().ctx; }

inline std::string data_dir() { return cm_data_dir(); }

}  // namespace cudamonsel

// ------------------------------------------------------------------ units and constants
namespace ToSI {
inline double eV(double e) { return e * 1.60217653e-19; }   // EPQLibrary/ToSI.cu:34-37
inline double keV(double e) { return e * 1.60217653e-16; }
}  // namespace ToSI
namespace FromSI {
inline double eV(double e) { return e * (1.0 / 1.60217653e-19); }
inline double keV(double e) { return e * (1.0 / 1.60217653e-16); }
}  // namespace FromSI
namespace Math2 {
constexpr double PI = 3.14159265358979323846;
}

// ------------------------------------------------------------------ elements and compositions
namespace Element {
class Element {
 public:
  explicit constexpr Element(int z = 0) : mZ(z) {}
  int getAtomicNumber() const { return mZ; }
  // atomic weights of EPQLibrary/AtomicWeights.csv as the reference reads them (std::stof)
  double getAtomicWeight() const {
    switch (mZ) {
      case 1: return (double)1.00794f;
      case 6: return (double)12.0107f;
      case 7: return (double)14.0067f;
      case 8: return (double)15.9994f;
      case 13: return (double)26.981538f;
      case 14: return (double)28.0855f;
      case 29: return (double)63.546f;
      case 79: return (double)196.96655f;
    }
    throw cudamonsel::Error(CM_EINVAL, "no NIST Mott data shipped for element " + std::to_string(mZ));
  }
  bool operator==(const Element& o) const { return mZ == o.mZ; }

 private:
  int mZ;
};
inline const Element H(1), C(6), N(7), O(8), Al(13), Si(14), Cu(29), Au(79);
inline const Element& byAtomicNumber(int z) {
  static const Element* all[] = {&H, &C, &N, &O, &Al, &Si, &Cu, &Au};
  for (const Element* e : all)
    if (e->getAtomicNumber() == z) return *e;
  throw cudamonsel::Error(CM_EINVAL, "no NIST Mott data shipped for element " + std::to_string(z));
}
}  // namespace Element
typedef Element::Element ElementT;

namespace Composition {
class Composition {
 public:
  // Composition::defineByMoleFraction: weight fraction of element i = n_i A_i / sum_j n_j A_j
  void defineByMoleFraction(const ElementT* elms[], int len, const double moleFracs[], int) {
    mElm.assign(elms, elms + len);
    double sum = 0;
    for (int i = 0; i < len; ++i) sum += moleFracs[i] * elms[i]->getAtomicWeight();
    mWf.resize(len);
    for (int i = 0; i < len; ++i) mWf[i] = moleFracs[i] * elms[i]->getAtomicWeight() / sum;
  }
  void defineByWeightFraction(const ElementT* elms[], int len, const double wf[], int) {
    mElm.assign(elms, elms + len);
    double sum = 0;
    for (int i = 0; i < len; ++i) sum += wf[i];
    mWf.resize(len);
    for (int i = 0; i < len; ++i) mWf[i] = wf[i] / sum;
  }
  std::vector<const ElementT*> mElm;
  std::vector<double> mWf;
};
}  // namespace Composition
typedef Composition::Composition CompositionT;

// ------------------------------------------------------------------ materials
namespace Material {
class Material {
 public:
  virtual ~Material() = default;
  CompositionT mComp;
  double mDensity = 0;
  std::string mName;
};
}  // namespace Material
typedef Material::Material MaterialT;

namespace SEmaterial {
class SEmaterial : public MaterialT {
 public:
  SEmaterial() = default;  // vacuum
  SEmaterial(const CompositionT& comp, double density) {
    mComp = comp;
    mDensity = density;
  }
  SEmaterial(const ElementT* elms[], int elemLen, const double weightFracs[], int wfLen, double density, const char* name) {
    mComp.defineByWeightFraction(elms, elemLen, weightFracs, wfLen);
    mDensity = density;
    mName = name ? name : "";
  }
  void setName(const std::string& n) { mName = n; }
  // SEmaterial::setWorkfunction keeps E_CB below -W (SEmaterial.cu:392-399)
  void setWorkfunction(double w) {
    mWork = w;
    if (mEcb > -w) mEcb = -w;
    cudamonsel::touch();
  }
  void setEnergyCBbottom(double e) { mEcb = e; cudamonsel::touch(); }
  void setBandgap(double g) { mGap = g; cudamonsel::touch(); }
  void setCoreEnergy(const double core[], int len) { mCore.assign(core, core + len); cudamonsel::touch(); }
  void addCoreEnergy(double e) { mCore.push_back(e); cudamonsel::touch(); }
  double getWorkfunction() const { return mWork; }
  double getEnergyCBbottom() const { return mEcb; }
  double getBandgap() const { return mGap; }
  double getEFermi() const { return -mEcb - mWork; }
  double mWork = 0, mEcb = 0, mGap = 0;
  std::vector<double> mCore;
};
}  // namespace SEmaterial
typedef SEmaterial::SEmaterial SEmaterialT;

// ------------------------------------------------------------------ mechanisms
namespace RandomizedScatterFactory {
class RandomizedScatterFactory {
 public:
  explicit constexpr RandomizedScatterFactory(int method) : mMethod(method) {}
  int mMethod;
};
}  // namespace RandomizedScatterFactory
typedef RandomizedScatterFactory::RandomizedScatterFactory RandomizedScatterFactoryT;

namespace NISTMottRS {  // JMONSEL/NISTMottRS.cu:506-512
inline const RandomizedScatterFactoryT Factory(1), Factory100(2), Factory100Lin(3);
}

namespace ScatterMechanism {
class ScatterMechanism {
 public:
  virtual ~ScatterMechanism() = default;
  virtual void realize(cm_context* ctx, int msm) const = 0;
};
}  // namespace ScatterMechanism
typedef ScatterMechanism::ScatterMechanism ScatterMechanismT;

namespace cudamonsel {
// NIST Mott tables of element Z into the context (E%02d.bin of the data directory)
inline void load_mott(cm_context* ctx, int z) {
  char name[32];
  snprintf(name, sizeof(name), "/NistXSec/E%02d.bin", z);
  const std::string path = data_dir() + name;
  std::ifstream f(path, std::ios::binary);
  char magic[8];
  int32_t head[4];
  if (!f.read(magic, 8) || memcmp(magic, "NMOTT001", 8) != 0 || !f.read((char*)head, sizeof(head)) || head[0] != z)
    throw Error(CM_EINVAL, "cannot read NIST Mott data " + path);
  std::vector<double> sp(head[1]), x1((size_t)head[1] * head[2]);
  f.read((char*)sp.data(), sp.size() * 8);
  f.read((char*)x1.data(), x1.size() * 8);
  if (!f) throw Error(CM_EINVAL, "truncated NIST Mott data " + path);
  check(cm_add_mott_element(ctx, z, sp.data(), x1.data()), "cm_add_mott_element");
}

// a NUTableInterpolation text table (JMONSEL/NUTableInterpolation.cu:117-228) into the context
inline int load_table(cm_context* ctx, const std::string& path) {
  std::ifstream f(path);
  if (!f) throw Error(CM_EINVAL, "cannot open table " + path);
  int dim = 0;
  f >> dim;
  if (!f || dim < 1 || dim > 3) throw Error(CM_EINVAL, "bad table " + path);
  std::vector<int> n(dim);
  std::vector<double> axes, vals;
  size_t total = 1;
  for (int k = 0; k < dim; ++k) {
    f >> n[k];
    if (!f || n[k] < 1) throw Error(CM_EINVAL, "bad table " + path);
    for (int i = 0; i < n[k]; ++i) {
      double x;
      f >> x;
      axes.push_back(x);
    }
    total *= (size_t)n[k];
  }
  vals.resize(total);
  for (size_t i = 0; i < total; ++i) f >> vals[i];
  if (!f) throw Error(CM_EINVAL, "truncated table " + path);
  int h = -1;
  check(cm_add_table(ctx, dim, n.data(), axes.data(), vals.data(), &h), "cm_add_table");
  return h;
}

// the build of one run: handles of the objects already replayed into the context
struct Build {
  cm_context* ctx;
  std::map<const void*, int> materials, msms;
  std::map<int, bool> motts;
  std::map<std::string, int> tables;
  int table(const std::string& p) {
    auto it = tables.find(p);
    if (it != tables.end()) return it->second;
    return tables[p] = load_table(ctx, p);
  }
  int material(const SEmaterialT& m) {
    auto it = materials.find(&m);
    if (it != materials.end()) return it->second;
    std::vector<int> z;
    std::vector<double> a, wf;
    for (size_t i = 0; i < m.mComp.mElm.size(); ++i) {
      z.push_back(m.mComp.mElm[i]->getAtomicNumber());
      a.push_back(m.mComp.mElm[i]->getAtomicWeight());
      wf.push_back(m.mComp.mWf[i]);
    }
    int h = -1;
    check(cm_add_material(ctx, (int)z.size(), z.data(), a.data(), wf.data(), m.mDensity, m.mWork, m.mEcb, m.mGap,
                          (int)m.mCore.size(), m.mCore.data(), &h),
          "cm_add_material");
    return materials[&m] = h;
  }
  void mott(int z) {
    if (!motts[z]) load_mott(ctx, z);
    motts[z] = true;
  }
};
thread_local inline Build* g_build = nullptr;
}  // namespace cudamonsel

namespace SelectableElasticSM {  // JMONSEL/SelectableElasticSM.cu:10-18
class SelectableElasticSM : public ScatterMechanismT {
 public:
  SelectableElasticSM(const MaterialT& mat, const RandomizedScatterFactoryT& f) : mMat(mat), mMethod(f.mMethod) {}
  void realize(cm_context* ctx, int msm) const override {
    for (const ElementT* e : mMat.mComp.mElm) cudamonsel::g_build->mott(e->getAtomicNumber());
    int h;
    cudamonsel::check(cm_msm_add_nistmott(ctx, msm, mMethod, &h), "cm_msm_add_nistmott");
  }
  const MaterialT& mMat;
  int mMethod;
};
}  // namespace SelectableElasticSM
typedef SelectableElasticSM::SelectableElasticSM SelectableElasticSMT;

namespace TabulatedInelasticSM {  // JMONSEL/TabulatedInelasticSM.cu:23-66
class TabulatedInelasticSM : public ScatterMechanismT {
 public:
  TabulatedInelasticSM(const SEmaterialT& mat, int methodSE, const StringT tables[], double energyOffset = 0.)
      : mMethodSE(methodSE), mOffset(energyOffset) {
    (void)mat;
    for (int k = 0; k < 4; ++k) mTables[k] = tables[k];
  }
  void realize(cm_context* ctx, int msm) const override {
    int t[4];
    for (int k = 0; k < 4; ++k) t[k] = cudamonsel::g_build->table(mTables[k]);
    int h;
    cudamonsel::check(cm_msm_add_tabulated(ctx, msm, mMethodSE, mOffset, t, &h), "cm_msm_add_tabulated");
  }
  int mMethodSE;
  double mOffset;
  StringT mTables[4];
};
}  // namespace TabulatedInelasticSM
typedef TabulatedInelasticSM::TabulatedInelasticSM TabulatedInelasticSMT;

namespace SlowingDownAlg {
class SlowingDownAlg {
 public:
  virtual ~SlowingDownAlg() = default;
  virtual void realize(cm_context* ctx, int msm) const = 0;
};
}  // namespace SlowingDownAlg
typedef SlowingDownAlg::SlowingDownAlg SlowingDownAlgT;

namespace JoyLuoNieminenCSD {  // JMONSEL/JoyLuoNieminenCSD.cu:42-121
class JoyLuoNieminenCSD : public SlowingDownAlgT {
 public:
  JoyLuoNieminenCSD(const SEmaterialT& mat, double breakE) : mBreakE(breakE) { (void)mat; }
  void realize(cm_context* ctx, int msm) const override {
    cudamonsel::check(cm_msm_set_csd_jln(ctx, msm, mBreakE), "cm_msm_set_csd_jln");
  }
  double mBreakE;
};
}  // namespace JoyLuoNieminenCSD
typedef JoyLuoNieminenCSD::JoyLuoNieminenCSD JoyLuoNieminenCSDT;

namespace FittedInelSM {  // JMONSEL/FittedInelSM.cu:8-25
class FittedInelSM : public ScatterMechanismT {
 public:
  FittedInelSM(const SEmaterialT& mat, double energySEgen, const JoyLuoNieminenCSDT& csd)
      : mE(energySEgen), mBreakE(csd.mBreakE) {
    (void)mat;
  }
  void realize(cm_context* ctx, int msm) const override {
    int h;
    cudamonsel::check(cm_msm_add_fitted(ctx, msm, mE, mBreakE, &h), "cm_msm_add_fitted");
  }
  double mE, mBreakE;
};
}  // namespace FittedInelSM
typedef FittedInelSM::FittedInelSM FittedInelSMT;

namespace GanachaudMokraniPolaronTrapSM {  // JMONSEL/GanachaudMokraniPolaronTrapSM.cu:8-27
class GanachaudMokraniPolaronTrapSM : public ScatterMechanismT {
 public:
  GanachaudMokraniPolaronTrapSM(double prefactor, double extinction) : mP(prefactor), mX(extinction) {}
  void realize(cm_context* ctx, int msm) const override {
    int h;
    cudamonsel::check(cm_msm_add_polaron(ctx, msm, mP, mX, &h), "cm_msm_add_polaron");
  }
  double mP, mX;
};
}  // namespace GanachaudMokraniPolaronTrapSM
typedef GanachaudMokraniPolaronTrapSM::GanachaudMokraniPolaronTrapSM GanachaudMokraniPolaronTrapSMT;

namespace GanachaudMokraniPhononInelasticSM {  // JMONSEL/GanachaudMokraniPhononInelasticSM.cu:8-72
class GanachaudMokraniPhononInelasticSM : public ScatterMechanismT {
 public:
  GanachaudMokraniPhononInelasticSM(double ratemult, double phononE, double temperature, double eps0, double epsInf)
      : a(ratemult), b(phononE), c(temperature), d(eps0), e(epsInf) {}
  void realize(cm_context* ctx, int msm) const override {
    int h;
    cudamonsel::check(cm_msm_add_phonon(ctx, msm, a, b, c, d, e, &h), "cm_msm_add_phonon");
  }
  double a, b, c, d, e;
};
}  // namespace GanachaudMokraniPhononInelasticSM
typedef GanachaudMokraniPhononInelasticSM::GanachaudMokraniPhononInelasticSM GanachaudMokraniPhononInelasticSMT;

namespace BarrierScatterMechanism {
class BarrierScatterMechanism {
 public:
  virtual ~BarrierScatterMechanism() = default;
  virtual void realize(cm_context* ctx, int msm) const = 0;
};
}  // namespace BarrierScatterMechanism
typedef BarrierScatterMechanism::BarrierScatterMechanism BarrierScatterMechanismT;

namespace ExpQMBarrierSM {  // JMONSEL/ExpQMBarrierSM.cu:12-28
class ExpQMBarrierSM : public BarrierScatterMechanismT {
 public:
  explicit ExpQMBarrierSM(const MaterialT* mat) : mClassical(true), mLambda(0) { (void)mat; }
  ExpQMBarrierSM(const MaterialT* mat, double lambda) : mClassical(lambda == 0), mLambda(lambda) { (void)mat; }
  void realize(cm_context* ctx, int msm) const override {
    cudamonsel::check(cm_msm_set_barrier(ctx, msm, mClassical ? 1 : 0, mLambda), "cm_msm_set_barrier");
  }
  bool mClassical;
  double mLambda;
};
}  // namespace ExpQMBarrierSM
typedef ExpQMBarrierSM::ExpQMBarrierSM ExpQMBarrierSMT;

// ------------------------------------------------------------------ material scatter models
namespace IMaterialScatterModel {
class IMaterialScatterModel {
 public:
  virtual ~IMaterialScatterModel() = default;
  virtual int realize(cudamonsel::Build& b) const = 0;
};
}  // namespace IMaterialScatterModel
typedef IMaterialScatterModel::IMaterialScatterModel IMaterialScatterModelT;

namespace MONSEL_MaterialScatterModel {  // JMONSEL/MONSEL_MaterialScatterModel.cu:13-162
class MONSEL_MaterialScatterModel : public IMaterialScatterModelT {
 public:
  MONSEL_MaterialScatterModel(const SEmaterialT* mat, const BarrierScatterMechanismT* barrier)
      : mMat(mat), mBarrier(barrier) {
    cudamonsel::touch();
  }
  void addScatterMechanism(const ScatterMechanismT* m) { mMech.push_back(m); cudamonsel::touch(); }
  void setCSD(const SlowingDownAlgT* csd) { mCsd = csd; cudamonsel::touch(); }
  void setMinEforTracking(double e) { mMinE = e; mMinESet = true; cudamonsel::touch(); }
  const SEmaterialT& getMaterial() const { return *mMat; }
  int realize(cudamonsel::Build& b) const override {
    auto it = b.msms.find(this);
    if (it != b.msms.end()) return it->second;
    int h = -1;
    cudamonsel::check(cm_add_msm(b.ctx, b.material(*mMat), &h), "cm_add_msm");
    for (const ScatterMechanismT* m : mMech) m->realize(b.ctx, h);
    if (mCsd) mCsd->realize(b.ctx, h);
    if (mBarrier) mBarrier->realize(b.ctx, h);
    if (mMinESet) cudamonsel::check(cm_msm_set_min_e(b.ctx, h, mMinE), "cm_msm_set_min_e");
    return b.msms[this] = h;
  }
  const SEmaterialT* mMat;
  const BarrierScatterMechanismT* mBarrier;
  std::vector<const ScatterMechanismT*> mMech;
  const SlowingDownAlgT* mCsd = nullptr;
  double mMinE = 0;
  bool mMinESet = false;
};
}  // namespace MONSEL_MaterialScatterModel
typedef MONSEL_MaterialScatterModel::MONSEL_MaterialScatterModel MONSEL_MaterialScatterModelT;

namespace NullMaterialScatterModel {  // NISTMonte/NullMaterialScatterModel.cu: vacuum without scattering
class NullMaterialScatterModel : public IMaterialScatterModelT {
 public:
  int realize(cudamonsel::Build& b) const override {
    auto it = b.msms.find(this);
    if (it != b.msms.end()) return it->second;
    int h = -1;
    cudamonsel::check(cm_add_msm(b.ctx, b.material(mVacuum), &h), "cm_add_msm");
    return b.msms[this] = h;
  }
  SEmaterialT mVacuum;
};
}  // namespace NullMaterialScatterModel
typedef NullMaterialScatterModel::NullMaterialScatterModel NullMaterialScatterModelT;

// ------------------------------------------------------------------ shapes
namespace Shape {
class Shape {
 public:
  virtual ~Shape() = default;
  // the shape, with the moves applied to it so far, as a new engine shape
  virtual int realize(cm_context* ctx) const = 0;

 protected:
  struct Move {
    bool rotate;
    double v[3], phi, theta, psi;
  };
  std::vector<Move> mMoves;
  int moved(cm_context* ctx, int h) const {
    for (const Move& m : mMoves) {
      if (m.rotate) cudamonsel::check(cm_shape_rotate(ctx, h, m.v, m.phi, m.theta, m.psi), "cm_shape_rotate");
      else cudamonsel::check(cm_shape_translate(ctx, h, m.v), "cm_shape_translate");
    }
    return h;
  }

 public:
  // ITransform
  void rotate(const double pivot[], double phi, double theta, double psi) {
    mMoves.push_back({true, {pivot[0], pivot[1], pivot[2]}, phi, theta, psi});
    cudamonsel::touch();
  }
  void translate(const double distance[]) {
    mMoves.push_back({false, {distance[0], distance[1], distance[2]}, 0, 0, 0});
    cudamonsel::touch();
  }
};
}  // namespace Shape
typedef Shape::Shape ShapeT;

namespace Sphere {  // NISTMonte/Sphere.cu
class Sphere : public ShapeT {
 public:
  Sphere(const double center[], double radius) : mR(radius) { memcpy(mC, center, sizeof(mC)); }
  int realize(cm_context* ctx) const override {
    int h;
    cudamonsel::check(cm_shape_sphere(ctx, mC, mR, &h), "cm_shape_sphere");
    return moved(ctx, h);
  }
  double mC[3], mR;
};
}  // namespace Sphere
typedef Sphere::Sphere SphereT;

namespace NormalShape {
class NormalShape : public ShapeT {};
}  // namespace NormalShape
typedef NormalShape::NormalShape NormalShapeT;

namespace Plane {  // NISTMonte/MultiPlaneShape.cu: Plane(normal, point)
class Plane {
 public:
  Plane(const double normal[], int, const double point[], int) {
    memcpy(mN, normal, sizeof(mN));
    memcpy(mP, point, sizeof(mP));
  }
  double mN[3], mP[3];
};
}  // namespace Plane
typedef Plane::Plane PlaneT;

namespace NormalMultiPlaneShape {  // JMONSEL/NormalMultiPlaneShape.cu
class NormalMultiPlaneShape : public NormalShapeT {
 public:
  void addPlane(const PlaneT& p) {
    mN.insert(mN.end(), p.mN, p.mN + 3);
    mP.insert(mP.end(), p.mP, p.mP + 3);
    cudamonsel::touch();
  }
  void addPlane(const double normal[], const double point[]) { addPlane(PlaneT(normal, 3, point, 3)); }
  int getNumPlanes() const { return (int)mN.size() / 3; }
  int realize(cm_context* ctx) const override {
    int h;
    cudamonsel::check(cm_shape_planes(ctx, getNumPlanes(), mN.data(), mP.data(), &h), "cm_shape_planes");
    return moved(ctx, h);
  }
  std::vector<double> mN, mP;
};
}  // namespace NormalMultiPlaneShape
typedef NormalMultiPlaneShape::NormalMultiPlaneShape NormalMultiPlaneShapeT;

namespace cudamonsel {
// shapes that read the options when they are built (cylinders, rounded lines) get the ones set then
template <typename F> int with_options(cm_context* ctx, int options, F make) {
  const int now = Session::state().options;
  check(cm_set_options(ctx, options), "cm_set_options");
  const int h = make();
  check(cm_set_options(ctx, now), "cm_set_options");
  return h;
}
}  // namespace cudamonsel

namespace NormalCylindricalShape {  // JMONSEL/NormalCylindricalShape.cu
class NormalCylindricalShape : public NormalShapeT {
 public:
  NormalCylindricalShape(const double end0[], const double end1[], double radius)
      : mR(radius), mOptions(cudamonsel::Session::state().options) {
    memcpy(mE0, end0, sizeof(mE0));
    memcpy(mE1, end1, sizeof(mE1));
  }
  int realize(cm_context* ctx) const override {
    const int h = cudamonsel::with_options(ctx, mOptions, [&] {
      int k;
      cudamonsel::check(cm_shape_cylinder(ctx, mE0, mE1, mR, &k), "cm_shape_cylinder");
      return k;
    });
    return moved(ctx, h);
  }
  double mE0[3], mE1[3], mR;
  int mOptions;
};
}  // namespace NormalCylindricalShape
typedef NormalCylindricalShape::NormalCylindricalShape NormalCylindricalShapeT;

namespace NormalIntersectionShape {  // JMONSEL/NormalIntersectionShape.cu
class NormalIntersectionShape : public NormalShapeT {
 public:
  NormalIntersectionShape(const NormalShapeT& a, const NormalShapeT& b) : mA(a), mB(b) {}
  int realize(cm_context* ctx) const override {
    int h;
    cudamonsel::check(cm_shape_intersection(ctx, mA.realize(ctx), mB.realize(ctx), &h), "cm_shape_intersection");
    return moved(ctx, h);
  }
  const NormalShapeT& mA;
  const NormalShapeT& mB;
};
}  // namespace NormalIntersectionShape
typedef NormalIntersectionShape::NormalIntersectionShape NormalIntersectionShapeT;

namespace NormalUnionShape {  // JMONSEL/NormalUnionShape.cu
class NormalUnionShape : public NormalShapeT {
 public:
  NormalUnionShape(const NormalShapeT& a, const NormalShapeT& b) : mA(a), mB(b) {}
  int realize(cm_context* ctx) const override {
    int h;
    cudamonsel::check(cm_shape_union(ctx, mA.realize(ctx), mB.realize(ctx), &h), "cm_shape_union");
    return moved(ctx, h);
  }
  const NormalShapeT& mA;
  const NormalShapeT& mB;
};
}  // namespace NormalUnionShape
typedef NormalUnionShape::NormalUnionShape NormalUnionShapeT;

namespace NShapes {  // JMONSEL/NShapes.cu:55-149
class Line : public NormalIntersectionShapeT {
 public:
  Line(double topz, double width, double length, double thetal, double thetar, double radl, double radr)
      : NormalIntersectionShapeT(*this, *this), a{topz, width, length, thetal, thetar, radl, radr},
        mOptions(cudamonsel::Session::state().options) {}
  int realize(cm_context* ctx) const override {
    const int h = cudamonsel::with_options(ctx, mOptions, [&] {
      int k;
      cudamonsel::check(cm_shape_line(ctx, a[0], a[1], a[2], a[3], a[4], a[5], a[6], &k), "cm_shape_line");
      return k;
    });
    return moved(ctx, h);
  }
  double a[7];
  int mOptions;
};
// the line is an intersection of plane sets (with unions of a plane set and a cylinder at rounded corners);
// like the reference's, it lives until the process ends
inline NormalShapeT* createLine(double topz, double width, double length, double thetal, double thetar,
                                double radl = 0., double radr = 0.) {
  return new Line(topz, width, length, thetal, thetar, radl, radr);
}
}  // namespace NShapes

// ------------------------------------------------------------------ regions
namespace RegionBase {
class Region {
 public:
  Region(Region* parent, const IMaterialScatterModelT* msm, const ShapeT* shape)
      : mParent(parent), mMsm(msm), mShape(shape) {
    if (parent) parent->mSub.push_back(this);
    cudamonsel::touch();
  }
  ~Region() {
    if (mParent) {
      auto& v = mParent->mSub;
      for (size_t i = 0; i < v.size(); ++i)
        if (v[i] == this) v.erase(v.begin() + i--);
    }
    cudamonsel::touch();
  }
  // RegionBase::updateMaterial (NISTMonte/RegionBase.cu:21-28): replace a scatter model here and below
  void updateMaterial(const IMaterialScatterModelT& oldMsm, const IMaterialScatterModelT& newMsm) {
    if (mMsm == &oldMsm) mMsm = &newMsm;
    for (Region* r : mSub) r->updateMaterial(oldMsm, newMsm);
    cudamonsel::touch();
  }
  const IMaterialScatterModelT* getScatterModel() const { return mMsm; }
  void removeSubRegion(Region& r) {
    for (size_t i = 0; i < mSub.size(); ++i)
      if (mSub[i] == &r) mSub.erase(mSub.begin() + i--);
    cudamonsel::touch();
  }
  // this region and its subregions into the engine (parents first, subregions in the order they were added)
  void realize(cudamonsel::Build& b, int parent, int* out) const {
    int h;
    cudamonsel::check(cm_region_add(b.ctx, parent, mMsm->realize(b), mShape->realize(b.ctx), &h), "cm_region_add");
    if (out) *out = h;
    for (const Region* r : mSub) r->realize(b, h, nullptr);
  }
  Region* mParent;
  const IMaterialScatterModelT* mMsm;
  const ShapeT* mShape;
  std::vector<Region*> mSub;
};
}  // namespace RegionBase
typedef RegionBase::Region RegionT;

// ------------------------------------------------------------------ beam, listeners, the Monte Carlo
namespace Electron {
class Electron {};
}  // namespace Electron
typedef Electron::Electron ElectronT;

namespace ElectronGun {
class ElectronGun {
 public:
  virtual ~ElectronGun() = default;
  virtual void setBeamEnergy(double e) = 0;
  virtual double getBeamEnergy() const = 0;
  virtual void setCenter(const double center[]) = 0;
  virtual const double* getCenter() const = 0;
  virtual double getWidth() const = 0;
};
}  // namespace ElectronGun
typedef ElectronGun::ElectronGun ElectronGunT;

namespace GaussianBeam {  // NISTMonte/GaussianBeam.cu:20-65
class GaussianBeam : public ElectronGunT {
 public:
  GaussianBeam(double width, double energy, const double center[]) : mWidth(width), mE(energy) {
    memcpy(mC, center, sizeof(mC));
  }
  void setBeamEnergy(double e) override { mE = e; }
  double getBeamEnergy() const override { return mE; }
  void setCenter(const double center[]) override { memcpy(mC, center, sizeof(mC)); }
  const double* getCenter() const override { return mC; }
  void setWidth(double w) { mWidth = w; }
  double getWidth() const override { return mWidth; }
  // the engine starts its electrons itself; MonteCarloSS takes this one and ignores it
  ElectronT* createElectron() const {
    static ElectronT e;
    return &e;
  }
  double mWidth, mE, mC[3];
};
}  // namespace GaussianBeam
typedef GaussianBeam::GaussianBeam GaussianBeamT;

namespace Histogram {  // Utility/Histogram.cu:25-137
class Histogram {
 public:
  Histogram(double min, double max, int nBins) : mMin(min), mMax(max), mN(nBins), mCounts(nBins + 2, 0) {}
  int binCount() const { return mN; }
  int counts(int bin) const { return (int)mCounts[bin + 1]; }  // bin -1: below, binCount(): above
  int totalCounts() const {
    int s = 0;
    for (int64_t c : mCounts) s += (int)c;
    return s;
  }
  double minValue(int bin) const { return bin > -1 ? (bin == 0 ? mMin : mMin + bin * ((mMax - mMin) / mN)) : -INFINITY; }
  double maxValue(int bin) const { return bin + 1 <= mN ? mMin + (bin + 1) * ((mMax - mMin) / mN) : INFINITY; }
  void clear() { std::fill(mCounts.begin(), mCounts.end(), 0); }
  double mMin, mMax;
  int mN;
  std::vector<int64_t> mCounts;
};
}  // namespace Histogram
typedef Histogram::Histogram HistogramT;

namespace ActionListener {
class ActionListener {
 public:
  virtual ~ActionListener() = default;
  virtual void actionPerformed(const int) {}
};
}  // namespace ActionListener
typedef ActionListener::ActionListener ActionListenerT;

namespace MonteCarloSS { class MonteCarloSS; }
typedef MonteCarloSS::MonteCarloSS MonteCarloSST;

namespace BackscatterStats {  // NISTMonte/BackscatterStats.cu:94-255
class BackscatterStats : public ActionListenerT {
 public:
  inline explicit BackscatterStats(const MonteCarloSST& mcss, int nEnergyBins = 400);
  const HistogramT& backscatterEnergyHistogram() const { return mBack; }
  const HistogramT& forwardscatterEnergyHistogram() const { return mFwd; }
  const HistogramT& elevationHistogram() const { return mElev; }
  const HistogramT& azimuthalHistogram() const { return mAzim; }
  double backscatterFraction() const { return (double)mBack.totalCounts() / (double)mEventCount; }
  double forwardscatterFraction() const { return (double)mFwd.totalCounts() / (double)mEventCount; }
  double scatterFraction() const { return backscatterFraction() + forwardscatterFraction(); }
  int getEnergyBinCount() const { return mBins; }
  int mBins;
  double mBeamEnergy;  // eV
  HistogramT mBack, mFwd, mElev, mAzim;
  int mEventCount = 0;
};
}  // namespace BackscatterStats
typedef BackscatterStats::BackscatterStats BackscatterStatsT;

namespace MonteCarloSS {  // NISTMonte/MonteCarloSS.cu:28-231
class MonteCarloSS {
 public:
  static constexpr double ChamberRadius = 0.1;
  MonteCarloSS(ElectronGunT* gun, RegionT* chamber, ElectronT*) : mGun(gun), mChamber(chamber) {}
  double getBeamEnergy() const { return mGun->getBeamEnergy(); }
  ElectronGunT* getElectronGun() const { return mGun; }
  void setElectronGun(ElectronGunT* g) { mGun = g; }
  void addActionListener(ActionListenerT& l) { mListeners.push_back(&l); }
  void removeActionListener(ActionListenerT& l) {
    for (size_t i = 0; i < mListeners.size(); ++i)
      if (mListeners[i] == &l) mListeners.erase(mListeners.begin() + i--);
  }
  // n trajectories from the gun into the chamber, tallied by every BackscatterStats listening
  void runMultipleTrajectories(int n) {
    cudamonsel::Session& s = cudamonsel::Session::get();
    if (s.version != mBuilt || s.ctx != mCtx) {
      check_rebuild(s);
    }
    std::vector<BackscatterStatsT*> stats;
    for (ActionListenerT* l : mListeners)
      if (auto* b = dynamic_cast<BackscatterStatsT*>(l)) stats.push_back(b);
    const int nb = stats.empty() ? 1 : stats[0]->mBins;
    for (size_t k = 0; k < std::max<size_t>(1, stats.size()); ++k) {
      BackscatterStatsT* st = stats.empty() ? nullptr : stats[k];
      const int bins = st ? st->mBins : nb;
      const double* c = mGun->getCenter();
      const double E = mGun->getBeamEnergy();
      cm_run_desc d;
      memset(&d, 0, sizeof(d));
      d.chamber = mChamberHandle;
      d.precision = s.precision;
      d.npix = 1;
      d.beam_width = mGun->getWidth();
      d.pixel_center = c;
      d.pixel_energy = &E;
      d.pixel_nprim = &n;
      d.pixel_nbins = &bins;
      d.seed = s.seed + s.runs++;
      d.hist_stride = bins + 2;
      std::vector<uint32_t> back(bins + 2), fwd(bins + 2), elev(CM_ELEVATION_COUNTS), azim(CM_AZIMUTH_COUNTS);
      if (st) {
        d.elevation = elev.data();
        d.azimuth = azim.data();
      }
      cm_run_stats rs;
      cudamonsel::check(cm_run(s.ctx, &d, back.data(), fwd.data(), &rs), "cm_run");
      if (st) {
        for (int i = 0; i < bins + 2; ++i) {
          st->mBack.mCounts[i] += back[i];
          st->mFwd.mCounts[i] += fwd[i];
        }
        for (int i = 0; i < CM_ELEVATION_COUNTS; ++i) st->mElev.mCounts[i] += elev[i];
        for (int i = 0; i < CM_AZIMUTH_COUNTS; ++i) st->mAzim.mCounts[i] += azim[i];
        st->mEventCount += n;
      }
    }
  }
  RegionT* getChamber() const { return mChamber; }
  int chamberHandle() const { return mChamberHandle; }

 private:
  void check_rebuild(cudamonsel::Session& s) {
    cudamonsel::check(cm_context_reset(s.ctx), "cm_context_reset");
    cudamonsel::check(cm_set_options(s.ctx, s.options), "cm_set_options");
    cudamonsel::Build b{s.ctx};
    cudamonsel::g_build = &b;
    try {
      mChamber->realize(b, -1, &mChamberHandle);
    } catch (...) {
      cudamonsel::g_build = nullptr;
      throw;
    }
    cudamonsel::g_build = nullptr;
    mBuilt = s.version;
    mCtx = s.ctx;
  }
  ElectronGunT* mGun;
  RegionT* mChamber;
  int mChamberHandle = -1;
  unsigned long long mBuilt = 0;
  cm_context* mCtx = nullptr;
  std::vector<ActionListenerT*> mListeners;
};
}  // namespace MonteCarloSS

inline BackscatterStats::BackscatterStats::BackscatterStats(const MonteCarloSST& mcss, int nEnergyBins)
    : mBins(nEnergyBins), mBeamEnergy(FromSI::eV(mcss.getBeamEnergy())), mBack(0.0, mBeamEnergy, nEnergyBins),
      mFwd(0.0, mBeamEnergy, nEnergyBins), mElev(0.0, Math2::PI, 180), mAzim(0.0, 2.0 * Math2::PI, 360) {}

#endif  // CUDAMONSEL_B200_HPP
