// Driver for the reference's own CPU transport code (CudaMONSEL, compiled out of
// tree by oracle/build_ref.py).  Test infrastructure only: it writes the golden
// vectors under tests/golden/ and runs whole trajectories for the statistical
// checks and the CPU timing.  It calls the reference's public classes exactly
// as its own driver does (JMONSELTests/LinesOnLayers.cu:80-282) and injects
// uniform deviates through the Math2::random() hook.
//
//   ref_driver golden <outdir> <SiTablesDir>
//   ref_driver golden2 <outdir>                  (sets added later: rotated shapes)
//   ref_driver run1 <nprim> <seed> <SiTablesDir> [beam_eV]
//   ref_driver run2 <nprim_per_px> <seed> <SiTablesDir> <x0_nm> <dx_nm> <npix> [beam_eV]
//   ref_driver scene <scene.txt> <pixels.txt> <seed> <beam_width_m> [angles]
//     (scene.txt from cudamonsel_b200.scenes.SceneSpec.to_text; pixels.txt rows: x y z [m] E [J] nprim nbins)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <deque>
#include <random>
#include <string>
#include <vector>

#include "gov/nist/microanalysis/EPQLibrary/Element.cuh"
#include "gov/nist/microanalysis/EPQLibrary/Material.cuh"
#include "gov/nist/microanalysis/EPQLibrary/Composition.cuh"
#include "gov/nist/microanalysis/EPQLibrary/ToSI.cuh"
#include "gov/nist/microanalysis/EPQLibrary/FromSI.cuh"
#include "gov/nist/microanalysis/EPQLibrary/NISTMottScatteringAngle.cuh"
#include "gov/nist/microanalysis/EPQLibrary/MeanIonizationPotential.cuh"
#include "gov/nist/microanalysis/EPQLibrary/CzyzewskiMottScatteringAngle.cuh"
#include "gov/nist/microanalysis/EPQLibrary/GasScatteringCrossSection.cuh"
#include "gov/nist/microanalysis/EPQLibrary/RandomizedScatter.cuh"
#include "gov/nist/microanalysis/NISTMonte/Electron.cuh"
#include "gov/nist/microanalysis/NISTMonte/MonteCarloSS.cuh"
#include "gov/nist/microanalysis/NISTMonte/GaussianBeam.cuh"
#include "gov/nist/microanalysis/NISTMonte/Sphere.cuh"
#include "gov/nist/microanalysis/NISTMonte/RegionBase.cuh"
#include "gov/nist/microanalysis/NISTMonte/MultiPlaneShape.cuh"
#include "gov/nist/microanalysis/NISTMonte/NullMaterialScatterModel.cuh"
#include "gov/nist/microanalysis/NISTMonte/BackscatterStats.cuh"
#include "gov/nist/microanalysis/Utility/Histogram.cuh"
#include "gov/nist/microanalysis/Utility/ActionListener.cuh"
#include "gov/nist/microanalysis/Utility/Math2.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/SEmaterial.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/ExpQMBarrierSM.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/MONSEL_MaterialScatterModel.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/SelectableElasticSM.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/NISTMottRS.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/TabulatedInelasticSM.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/NUTableInterpolation.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/JoyLuoNieminenCSD.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/FittedInelSM.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/GanachaudMokraniPolaronTrapSM.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/GanachaudMokraniPhononInelasticSM.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/NormalMultiPlaneShape.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/NormalIntersectionShape.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/NShapes.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/NormalCylindricalShape.cuh"
#include "gov/nist/nanoscalemetrology/JMONSEL/NormalUnionShape.cuh"

// ---------------------------------------------------------------- deviate hook
static std::deque<double> g_queue;
static std::mt19937_64 g_gen(0);
static long long g_drawn = 0;

extern "C" double cm_ref_uniform(void)
{
   ++g_drawn;
   if (!g_queue.empty()) {
      double u = g_queue.front();
      g_queue.pop_front();
      return u;
   }
   return (double)(g_gen() >> 11) * (1.0 / 9007199254740992.0);
}

static void push(std::initializer_list<double> us)
{
   g_queue.clear();
   for (double u : us) g_queue.push_back(u);
   g_drawn = 0;
}

// deterministic input generator for the golden sets (independent of the hook)
static std::mt19937_64 g_in(12345);
static double uin() { return (double)(g_in() >> 11) * (1.0 / 9007199254740992.0); }

static void init_reference()
{
   CzyzewskiMottScatteringAngle::init();
   NISTMottScatteringAngle::init();
   GasScatteringCrossSection::init();
   NISTMottRS::init();
   MeanIonizationPotential::Berger64MeanIonizationPotential::readTabulatedValues();
   MeanIonizationPotential::Berger83MeanIonizationPotential::readTabulatedValues();
}

// ---------------------------------------------------------------- materials as LinesOnLayers.cu builds them
struct SiModel {
   SEmaterialT* SiMat;
   StringT tables[4];
   SelectableElasticSMT* el;
   TabulatedInelasticSMT* inel;
   ExpQMBarrierSMT* barrier;
   MONSEL_MaterialScatterModelT* msm;
   SiModel(const std::string&)
   {
      const ElementT* comp[] = { &Element::Si };
      const double frac[] = { 1. };
      SiMat = new SEmaterialT(comp, 1, frac, 1, 2330., (char*)"Silicon");
      SiMat->setWorkfunction(ToSI::eV(4.85));
      SiMat->setEnergyCBbottom(ToSI::eV(-4.85 - (-1.1)));
      SiMat->setBandgap(ToSI::eV(1.1));
      double core[] = { ToSI::eV(99.2), ToSI::eV(99.8), ToSI::eV(149.7), ToSI::eV(1839.) };
      SiMat->setCoreEnergy(core, 4);
   }
   void build(const std::string& dir)
   {
      tables[0] = dir + "/IIMFPFullPennInterpSiSI.csv";
      tables[1] = dir + "/interpNUSimReducedDeltaEFullPennSiSI.csv";
      tables[2] = dir + "/interpNUThetaFullPennSiBGSI.csv";
      tables[3] = dir + "/interpSimESE0NUSiBGSI.csv";
      el = new SelectableElasticSMT(*SiMat, NISTMottRS::Factory);
      inel = new TabulatedInelasticSMT(*SiMat, 3, tables, ToSI::eV(13.54));
      barrier = new ExpQMBarrierSMT(SiMat);
      msm = new MONSEL_MaterialScatterModelT(SiMat, barrier);
      msm->addScatterMechanism(el);
      msm->addScatterMechanism(inel);
   }
};

struct PMMAModel {
   SEmaterialT* PMMA;
   SelectableElasticSMT* el;
   JoyLuoNieminenCSDT* csd;
   FittedInelSMT* fitted;
   GanachaudMokraniPolaronTrapSMT* polaron;
   ExpQMBarrierSMT* barrier;
   MONSEL_MaterialScatterModelT* msm;
   void build()
   {
      const ElementT* comp[] = { &Element::C, &Element::O, &Element::H };
      const double mol[] = { 5, 2, 8 };
      CompositionT c;
      c.defineByMoleFraction(comp, 3, mol, 3);
      PMMA = new SEmaterialT(c, 1190.);
      PMMA->setName("PMMA");
      PMMA->setWorkfunction(ToSI::eV(5.5));
      PMMA->setBandgap(ToSI::eV(5.));
      PMMA->setEnergyCBbottom(ToSI::eV(-5.5 - (-5.)));
      el = new SelectableElasticSMT(*PMMA, NISTMottRS::Factory);
      csd = new JoyLuoNieminenCSDT(*PMMA, ToSI::eV(45.));
      fitted = new FittedInelSMT(*PMMA, ToSI::eV(65.4), *csd);
      polaron = new GanachaudMokraniPolaronTrapSMT(2.e7, 1. / ToSI::eV(4.));
      barrier = new ExpQMBarrierSMT(PMMA);
      msm = new MONSEL_MaterialScatterModelT(PMMA, barrier);
      msm->addScatterMechanism(el);
      msm->addScatterMechanism(fitted);
      msm->addScatterMechanism(polaron);
      msm->setCSD(csd);
   }
};

static FILE* openw(const std::string& dir, const char* name)
{
   std::string p = dir + "/" + name;
   FILE* f = fopen(p.c_str(), "w");
   if (!f) { perror(p.c_str()); exit(2); }
   return f;
}

#define G "%.17g"

// NShapes::createLine (radius 0) with every plane point moved by dx along x.
// The reference's NormalIntersectionShape::translate (NormalIntersectionShape.cu:257-263)
// casts its children to the unrelated ITransform class and crashes, so a line
// away from x = 0 is assembled here from the same public classes instead; the
// plane points are computed as Plane::translate would (point[0] + dx).
static NormalIntersectionShapeT* make_line(double topz, double width, double length, double thetal, double thetar, double dx)
{
   NormalMultiPlaneShapeT* enclosure = new NormalMultiPlaneShapeT();
   double signz = !topz ? 0 : (topz > 0 ? 1 : -1);
   if (signz == 0.) signz = 1.;
   double n0[] = { 0., 0., signz }, p0[] = { 0. + dx, 0., topz };
   enclosure->addPlane(*new PlaneT(n0, 3, p0, 3));
   double n1[] = { 0., 0., -signz }, p1[] = { 0. + dx, 0., 0. };
   enclosure->addPlane(*new PlaneT(n1, 3, p1, 3));
   double n2[] = { 0., 1., 0. }, p2[] = { 0. + dx, length / 2., 0. };
   enclosure->addPlane(*new PlaneT(n2, 3, p2, 3));
   double n3[] = { 0., -1., 0. }, p3[] = { 0. + dx, -length / 2., 0. };
   enclosure->addPlane(*new PlaneT(n3, 3, p3, 3));
   NormalMultiPlaneShapeT* rightNMPS = new NormalMultiPlaneShapeT();
   double costhetar = ::cos(thetar), sinthetar = ::sin(thetar);
   double n4[] = { costhetar, 0., signz * sinthetar }, p4[] = { width / 2 + dx, 0., 0. };
   rightNMPS->addPlane(*new PlaneT(n4, 3, p4, 3));
   NormalMultiPlaneShapeT* leftNMPS = new NormalMultiPlaneShapeT();
   double costhetal = ::cos(thetal), sinthetal = ::sin(thetal);
   double n6[] = { -costhetal, 0., signz * sinthetal }, p6[] = { -width / 2 + dx, 0., 0. };
   leftNMPS->addPlane(*new PlaneT(n6, 3, p6, 3));
   NormalIntersectionShapeT* nts = new NormalIntersectionShapeT(*leftNMPS, *rightNMPS);
   return new NormalIntersectionShapeT(*nts, *enclosure);
}

// ---------------------------------------------------------------- golden sets
static void golden_nistmott(const std::string& out)
{
   FILE* f = openw(out, "nistmott.txt");
   fprintf(f, "# NISTMottRS (method 1) totalCrossSection and randomScatteringAngle; energies in J, sigma in m^2\n");
   fprintf(f, "# Z E u1 u2 sigma theta ndeviates\n");
   const int Zs[] = { 1, 6, 8, 14, 29, 79 };
   std::vector<double> Es;
   for (int i = 0; i < 400; ++i) Es.push_back(ToSI::eV(::exp(::log(1.0) + (::log(30000.0) - ::log(1.0)) * uin())));
   for (int k = 0; k <= 60; ++k) Es.push_back(::exp(::log(ToSI::keV(0.05)) + k * (::log(ToSI::keV(20.)) - ::log(ToSI::keV(0.05))) / 60.0));
   Es.push_back(ToSI::eV(50.)); Es.push_back(ToSI::keV(20.)); Es.push_back(ToSI::eV(49.999)); Es.push_back(ToSI::eV(1.)); Es.push_back(ToSI::eV(3.75));
   for (int z : Zs) {
      const RandomizedScatterT& rs = NISTMottRS::Factory.get(Element::byAtomicNumber(z));
      for (size_t i = 0; i < Es.size(); ++i) {
         double E = Es[i];
         double u1 = uin(), u2 = uin();
         if (i % 37 == 0) u1 = 0.0;
         if (i % 41 == 0) u1 = 1.0;
         if (i % 43 == 0) u2 = 1.0;
         double sigma = rs.totalCrossSection(E);
         push({ u1, u2 });
         double th = rs.randomScatteringAngle(E);
         fprintf(f, "%d " G " " G " " G " " G " " G " %lld\n", z, E, u1, u2, sigma, th, g_drawn);
      }
   }
   fclose(f);
}

// NISTMottRS methods 2 (Factory100: Browning below 100 eV) and 3 (Factory100Lin: linear below 100 eV)
static void golden_nistmott23(const std::string& out)
{
   FILE* f = openw(out, "nistmott23.txt");
   fprintf(f, "# NISTMottRS methods 2 and 3 totalCrossSection and randomScatteringAngle; energies in J, sigma in m^2\n");
   fprintf(f, "# method Z E u1 u2 sigma theta ndeviates\n");
   const int Zs[] = { 1, 6, 8, 14, 29, 79 };
   std::vector<double> Es;
   for (int i = 0; i < 300; ++i) Es.push_back(ToSI::eV(::exp(::log(1.0) + (::log(30000.0) - ::log(1.0)) * uin())));
   for (int i = 0; i < 100; ++i) Es.push_back(ToSI::eV(40.0 + 80.0 * uin()));
   Es.push_back(ToSI::eV(100.)); Es.push_back(ToSI::eV(99.999)); Es.push_back(ToSI::eV(50.)); Es.push_back(ToSI::eV(49.999));
   Es.push_back(ToSI::keV(20.)); Es.push_back(ToSI::eV(1.)); Es.push_back(ToSI::eV(3.75));
   for (int method = 2; method <= 3; ++method) {
      const RandomizedScatterFactoryT& fac = method == 2 ? NISTMottRS::Factory100 : NISTMottRS::Factory100Lin;
      for (int z : Zs) {
         const RandomizedScatterT& rs = fac.get(Element::byAtomicNumber(z));
         for (size_t i = 0; i < Es.size(); ++i) {
            double E = Es[i];
            double u1 = uin(), u2 = uin();
            if (i % 37 == 0) u1 = 0.0;
            if (i % 43 == 0) u2 = 1.0;
            double sigma = rs.totalCrossSection(E);
            push({ u1, u2 });
            double th = rs.randomScatteringAngle(E);
            fprintf(f, "%d %d " G " " G " " G " " G " " G " %lld\n", method, z, E, u1, u2, sigma, th, g_drawn);
         }
      }
   }
   fclose(f);
}

static void golden_nutable(const std::string& out, const SiModel& si)
{
   FILE* f = openw(out, "nutable.txt");
   fprintf(f, "# NUTableInterpolation::interpolate on the Si tables; table x0 x1 x2 order value\n");
   for (int t = 0; t < 4; ++t) {
      const NUTableInterpolationT* tab = NUTableInterpolation::getInstance(si.tables[t].c_str());
      MatrixXd dom = tab->getDomain();
      int dim = (int)dom.size();
      for (int i = 0; i < 600; ++i) {
         double x[3] = { 0, 0, 0 };
         for (int d = 0; d < dim; ++d) {
            double lo = dom[d][0], hi = dom[d][1];
            double u = uin();
            if (d == 0 && t != 3) {
               // energies: log-uniform, with some points just outside the domain
               double a = ::log(lo) - 0.05, b = ::log(hi) + 0.05;
               x[d] = ::exp(a + (b - a) * u);
            }
            else if (d == 0) {
               double a = ::log(lo), b = ::log(hi);
               x[d] = ::exp(a + (b - a) * u);
            }
            else x[d] = lo + (hi - lo) * u;
         }
         int orders[] = { 1, 3 };
         for (int order : orders) {
            if (t == 0 && order == 3) continue;
            if (t != 0 && order == 1) continue;
            double v = tab->interpolate(x, 3, order);
            fprintf(f, "%d " G " " G " " G " %d " G "\n", t, x[0], x[1], x[2], order, v);
         }
      }
      VectorXd range = tab->getRange();
      fprintf(f, "# range %d " G " " G "\n", t, range[0], range[1]);
   }
   fclose(f);
}

static void golden_tabinel(const std::string& out, SiModel& si)
{
   FILE* f = openw(out, "tabinel.txt");
   fprintf(f, "# TabulatedInelasticSM(Si, methodSE=3, offset=13.54 eV): scatterRate and scatter with injected deviates\n");
   fprintf(f, "# E theta phi u0..u5 rate | E' theta' phi' hasSE ESE thetaSE phiSE ndeviates\n");
   for (int i = 0; i < 3000; ++i) {
      double EeV = ::exp(::log(2.0) + (::log(15000.0) - ::log(2.0)) * uin());
      double E = ToSI::eV(EeV);
      double th = Math2::PI * uin(), ph = 2 * Math2::PI * uin() - Math2::PI;
      double u[6];
      for (int k = 0; k < 6; ++k) u[k] = uin();
      double pos[] = { 0, 0, 1e-8 };
      ElectronT e(pos, th, ph, E);
      double rate = si.inel->scatterRate(&e);
      push({ u[0], u[1], u[2], u[3], u[4], u[5] });
      ElectronT* se = si.inel->scatter(&e);
      fprintf(f, G " " G " " G, E, th, ph);
      for (int k = 0; k < 6; ++k) fprintf(f, " " G, u[k]);
      fprintf(f, " " G " " G " " G " " G " %d", rate, e.getEnergy(), e.getTheta(), e.getPhi(), se ? 1 : 0);
      if (se) fprintf(f, " " G " " G " " G, se->getEnergy(), se->getTheta(), se->getPhi());
      else fprintf(f, " 0 0 0");
      fprintf(f, " %lld\n", g_drawn);
      delete se;
   }
   fclose(f);
}

static void golden_elastic(const std::string& out, SiModel& si, PMMAModel& pm)
{
   FILE* f = openw(out, "elastic.txt");
   fprintf(f, "# SelectableElasticSM: material(0=Si,1=PMMA) E theta phi u0 u1 u2 rate theta' phi' Zscatter ndeviates\n");
   SelectableElasticSMT* sms[] = { si.el, pm.el };
   for (int m = 0; m < 2; ++m) {
      for (int i = 0; i < 1500; ++i) {
         double E = ToSI::eV(::exp(::log(1.0) + (::log(25000.0) - ::log(1.0)) * uin()));
         double th = Math2::PI * uin(), ph = 2 * Math2::PI * uin() - Math2::PI;
         double u0 = uin(), u1 = uin(), u2 = uin(), u3 = uin();
         double pos[] = { 0, 0, 0 };
         ElectronT e(pos, th, ph, E);
         double rate = sms[m]->scatterRate(&e);
         push({ u0, u1, u2, u3 });
         sms[m]->scatter(&e);
         fprintf(f, "%d " G " " G " " G " " G " " G " " G " " G " " G " " G " " G " %d %lld\n", m, E, th, ph, u0, u1, u2, u3, rate,
            e.getTheta(), e.getPhi(), e.getScatteringElement()->getAtomicNumber(), g_drawn);
      }
   }
   fclose(f);
}

static void golden_pmma(const std::string& out, PMMAModel& pm)
{
   FILE* f = openw(out, "pmma.txt");
   fprintf(f, "# PMMA: element iteration order, JoyLuoNieminenCSD::compute, FittedInelSM/polaron rates\n");
   fprintf(f, "order");
   for (auto el : pm.PMMA->getElementSet()) fprintf(f, " %d", el->getAtomicNumber());
   fprintf(f, "\n");
   for (auto el : pm.PMMA->getElementSet())
      fprintf(f, "wf %d " G " " G "\n", el->getAtomicNumber(), pm.PMMA->weightFraction(*el, true), el->getAtomicWeight());
   fprintf(f, "density " G "\n", pm.PMMA->getDensity());
   for (int i = 0; i < 2000; ++i) {
      double E = ToSI::eV(::exp(::log(0.2) + (::log(20000.0) - ::log(0.2)) * uin()));
      double len = ::exp(::log(1e-12) + (::log(1e-6) - ::log(1e-12)) * uin());
      double pos[] = { 0, 0, 0 };
      ElectronT e(pos, 0., 0., E);
      double csd = pm.csd->compute(len, &e);
      double rf = pm.fitted->scatterRate(&e);
      double rp = pm.polaron->scatterRate(&e);
      fprintf(f, "csd " G " " G " " G " " G " " G "\n", E, len, csd, rf, rp);
   }
   // FittedInelSM::scatter with deviates
   for (int i = 0; i < 200; ++i) {
      double E = ToSI::eV(100.0 + 400 * uin());
      double u0 = uin(), u1 = uin();
      double pos[] = { 0, 0, 0 };
      ElectronT e(pos, 0.3, 0.2, E);
      push({ u0, u1 });
      ElectronT* se = pm.fitted->scatter(&e);
      fprintf(f, "fitted " G " " G " " G " " G " " G " " G " %lld\n", E, u0, u1, se->getEnergy(), se->getTheta(), se->getPhi(), g_drawn);
      delete se;
   }
   fclose(f);
}

static void golden_phonon(const std::string& out)
{
   FILE* f = openw(out, "phonon.txt");
   fprintf(f, "# GanachaudMokraniPhononInelasticSM(3, 0.063 eV, 300 K, 11.7, 1): E theta phi u0 u1 rate E' theta' phi' Eprev' ndeviates\n");
   GanachaudMokraniPhononInelasticSMT ph(3., ToSI::eV(0.063), 300., 11.7, 1.);
   for (int i = 0; i < 1000; ++i) {
      double E = ToSI::eV(::exp(::log(0.03) + (::log(2000.0) - ::log(0.03)) * uin()));
      double th = Math2::PI * uin(), phi = 2 * Math2::PI * uin() - Math2::PI;
      double u0 = uin(), u1 = uin();
      double pos[] = { 0, 0, 0 };
      ElectronT e(pos, th, phi, E);
      double rate = ph.scatterRate(&e);
      push({ u0, u1 });
      ph.scatter(&e);
      fprintf(f, G " " G " " G " " G " " G " " G " " G " " G " " G " " G " %lld\n", E, th, phi, u0, u1, rate, e.getEnergy(), e.getTheta(), e.getPhi(), e.getPreviousEnergy(), g_drawn);
   }
   fclose(f);
}

static void golden_shapes(const std::string& out)
{
   FILE* f = openw(out, "shapes.txt");
   fprintf(f, "# shape(0 half-space,1 block,2 line at x=25nm,3 createLine at x=0) p0(3) p1(3) | nx ny nz u contains(p0)\n");
   // 0: half-space z >= 0 (LinesOnLayers layer plane)
   NormalMultiPlaneShapeT* half = new NormalMultiPlaneShapeT();
   double nz[] = { 0., 0., -1. }, o[] = { 0., 0., 0. };
   half->addPlane(*new PlaneT(nz, 3, o, 3));
   // 1: a 6-plane block 30 x 20 x 10 nm centred at (5, -3, 12) nm
   NormalMultiPlaneShapeT* block = new NormalMultiPlaneShapeT();
   double c[] = { 5e-9, -3e-9, 12e-9 }, h[] = { 15e-9, 10e-9, 5e-9 };
   for (int a = 0; a < 3; ++a)
      for (int s = -1; s <= 1; s += 2) {
         double n[] = { 0, 0, 0 }, p[] = { c[0], c[1], c[2] };
         n[a] = s;
         p[a] += s * h[a];
         block->addPlane(*new PlaneT(n, 3, p, 3));
      }
   // 2: the trapezoid line of NShapes::createLine(-100 nm, 40 nm, 1 um, 3 deg, 3 deg, 0, 0), translated by (25 nm, 0, 0)
   NormalIntersectionShapeT* line = make_line(-100e-9, 40e-9, 1e-6, 3 * Math2::PI / 180, 3 * Math2::PI / 180, 25e-9);
   NormalIntersectionShapeT* line0 = (NormalIntersectionShapeT*)NShapes::createLine(-100e-9, 40e-9, 1e-6, 3 * Math2::PI / 180, 3 * Math2::PI / 180, 0, 0);
   NormalShapeT* shapes[] = { half, block, line, line0 };
   for (int s = 0; s < 4; ++s) {
      for (int i = 0; i < 4000; ++i) {
         double p0[3], p1[3];
         for (int k = 0; k < 3; ++k) p0[k] = (uin() * 160 - 80) * 1e-9;
         if (s >= 2) { p0[2] = (uin() * 140 - 120) * 1e-9; }
         double len = ::exp(::log(0.05e-9) + (::log(200e-9) - ::log(0.05e-9)) * uin());
         double th = Math2::PI * uin(), ph = 2 * Math2::PI * uin();
         p1[0] = p0[0] + len * ::sin(th) * ::cos(ph);
         p1[1] = p0[1] + len * ::sin(th) * ::sin(ph);
         p1[2] = p0[2] + len * ::cos(th);
         VectorXd r = shapes[s]->getFirstNormal(p0, p1);
         int inside = ((ShapeT*)shapes[s])->contains(p0) ? 1 : 0;
         fprintf(f, "%d " G " " G " " G " " G " " G " " G " " G " " G " " G " " G " %d\n", s, p0[0], p0[1], p0[2], p1[0], p1[1], p1[2], r[0], r[1], r[2], r[3], inside);
      }
   }
   fclose(f);
}

// NormalCylindricalShape, NormalUnionShape and createLine with rounded corners
static void golden_shapes2(const std::string& out)
{
   FILE* f = openw(out, "shapes2.txt");
   fprintf(f, "# shape(0 oblique cylinder,1 cylinder along y,2 union(block, oblique cylinder),3 createLine radl 5 nm radr 8 nm,"
              "4 the oblique cylinder translated by (30, 0, -10) nm, 5-7 shapes 0-2 with the cylinder axis normalised) "
              "p0(3) p1(3) | nx ny nz u contains(p0) contains(p0,p1)\n");
   double e0[] = { -20e-9, -10e-9, 30e-9 }, e1[] = { 25e-9, 15e-9, 50e-9 };
   NormalCylindricalShapeT* cyl = new NormalCylindricalShapeT(e0, e1, 12e-9);
   double f0[] = { 10e-9, -500e-9, -30e-9 }, f1[] = { 10e-9, 500e-9, -30e-9 };
   NormalCylindricalShapeT* cyly = new NormalCylindricalShapeT(f0, f1, 8e-9);
   NormalMultiPlaneShapeT* block = new NormalMultiPlaneShapeT();
   double c[] = { 5e-9, -3e-9, 12e-9 }, h[] = { 15e-9, 10e-9, 5e-9 };
   for (int a = 0; a < 3; ++a)
      for (int sg = -1; sg <= 1; sg += 2) {
         double n[] = { 0, 0, 0 }, p[] = { c[0], c[1], c[2] };
         n[a] = sg;
         p[a] += sg * h[a];
         block->addPlane(*new PlaneT(n, 3, p, 3));
      }
   double e0b[] = { -20e-9, -10e-9, 30e-9 }, e1b[] = { 25e-9, 15e-9, 50e-9 };
   NormalCylindricalShapeT* cylb = new NormalCylindricalShapeT(e0b, e1b, 12e-9);
   NormalUnionShapeT* uni = new NormalUnionShapeT(*block, *cylb);
   const double th = 3 * Math2::PI / 180;
   NormalShapeT* rline = NShapes::createLine(-100e-9, 40e-9, 1e-6, th, th, 5e-9, 8e-9);
   // (translating composites is unsafe in the reference: its casts between the
   // ITransform and Shape bases; a cylinder translates itself)
   double e0t[] = { -20e-9, -10e-9, 30e-9 }, e1t[] = { 25e-9, 15e-9, 50e-9 };
   NormalCylindricalShapeT* cylt = new NormalCylindricalShapeT(e0t, e1t, 12e-9);
   double d[] = { 30e-9, 0., -10e-9 };
   cylt->translate(d);
   // the same cylinders with their axis normalised: an identity rotation about the
   // origin recomputes normalizedaxis from the (by then initialised) length
   const double zero[] = { 0., 0., 0. };
   NormalCylindricalShapeT* wcyl = new NormalCylindricalShapeT(e0, e1, 12e-9);
   wcyl->rotate(zero, 0., 0., 0.);
   NormalCylindricalShapeT* wcyly = new NormalCylindricalShapeT(f0, f1, 8e-9);
   wcyly->rotate(zero, 0., 0., 0.);
   NormalCylindricalShapeT* wcylb = new NormalCylindricalShapeT(e0b, e1b, 12e-9);
   wcylb->rotate(zero, 0., 0., 0.);
   NormalMultiPlaneShapeT* block2 = new NormalMultiPlaneShapeT();
   for (int a = 0; a < 3; ++a)
      for (int sg = -1; sg <= 1; sg += 2) {
         double n[] = { 0, 0, 0 }, p[] = { c[0], c[1], c[2] };
         n[a] = sg;
         p[a] += sg * h[a];
         block2->addPlane(*new PlaneT(n, 3, p, 3));
      }
   NormalUnionShapeT* wuni = new NormalUnionShapeT(*block2, *wcylb);
   NormalShapeT* shapes[] = { cyl, cyly, uni, rline, cylt, wcyl, wcyly, wuni };
   for (int s = 0; s < 8; ++s) {
      for (int i = 0; i < 4000; ++i) {
         double p0[3], p1[3];
         for (int k = 0; k < 3; ++k) p0[k] = (uin() * 120 - 60) * 1e-9;
         if (s >= 5) {  // start near the cylinders so that many steps cross them
            const double* a0 = s == 6 ? f0 : e0;
            const double* a1 = s == 6 ? f1 : e1;
            const double t = s == 6 ? 0.45 + 0.1 * uin() : uin();
            for (int k = 0; k < 3; ++k) p0[k] = a0[k] + t * (a1[k] - a0[k]) + (uin() * 40 - 20) * 1e-9;
         }
         if (s == 3) {
            p0[0] = (uin() * 100 - 50) * 1e-9;
            p0[2] = (uin() * 130 - 120) * 1e-9;
         }
         if (s == 4) p0[0] += 30e-9;
         double len = ::exp(::log(0.05e-9) + (::log(200e-9) - ::log(0.05e-9)) * uin());
         double th2 = Math2::PI * uin(), ph = 2 * Math2::PI * uin();
         p1[0] = p0[0] + len * ::sin(th2) * ::cos(ph);
         p1[1] = p0[1] + len * ::sin(th2) * ::sin(ph);
         p1[2] = p0[2] + len * ::cos(th2);
         VectorXd r = shapes[s]->getFirstNormal(p0, p1);
         int inside = ((ShapeT*)shapes[s])->contains(p0) ? 1 : 0;
         int inside2 = shapes[s]->contains(p0, p1) ? 1 : 0;
         fprintf(f, "%d " G " " G " " G " " G " " G " " G " " G " " G " " G " " G " %d %d\n", s, p0[0], p0[1], p0[2], p1[0], p1[1],
                 p1[2], r[0], r[1], r[2], r[3], inside, inside2);
      }
   }
   fclose(f);
}

static void golden_misc(const std::string& out, SiModel& si)
{
   FILE* f = openw(out, "misc.txt");
   fprintf(f, "# beam: width cx cy cz u0 u1 | x y z\n");
   for (int i = 0; i < 200; ++i) {
      double w = 1e-9 * uin() * 3;
      double cen[] = { (uin() - 0.5) * 1e-7, (uin() - 0.5) * 1e-7, -1.2e-7 };
      GaussianBeamT eg(w, ToSI::eV(500.), cen);
      double u0 = uin(), u1 = uin();
      push({ u0, u1 });
      ElectronT* e = eg.createElectron();
      VectorXd p = e->getPosition();
      fprintf(f, "beam " G " " G " " G " " G " " G " " G " " G " " G " " G "\n", w, cen[0], cen[1], cen[2], u0, u1, p[0], p[1], p[2]);
      delete e;
   }
   fprintf(f, "# hist: min max nbins value bin\n");
   for (int nb : { 100, 50, 7 }) {
      double E0 = nb * 10.0;
      HistogramT hist(0.0, E0, nb);
      for (int i = 0; i < 300; ++i) {
         double v = (uin() * 1.1 - 0.05) * E0;
         if (i % 10 == 0) v = 10.0 * (int)(uin() * nb);
         if (v > E0) v = E0;
         fprintf(f, "hist " G " " G " %d " G " %d\n", 0.0, E0, nb, v, hist.bin(v));
      }
   }
   fprintf(f, "# msm (Si): E u | freepath ; E u_path u_mech -> mechanism index\n");
   for (int i = 0; i < 500; ++i) {
      double E = ToSI::eV(::exp(::log(4.0) + (::log(15000.0) - ::log(4.0)) * uin()));
      double u = uin();
      double pos[] = { 0, 0, 0 };
      ElectronT e(pos, 0.1, 0.2, E);
      push({ u });
      double fp = si.msm->randomMeanPathLength(e);
      fprintf(f, "fpath " G " " G " " G "\n", E, u, fp);
   }
   fclose(f);
}

struct ScatterCounter : public ActionListenerT {
   long long scatters = 0, nonscatters = 0, secondaries = 0;
   void actionPerformed(const int ae) override
   {
      if (ae == MonteCarloSS::ScatterEvent) ++scatters;
      else if (ae == MonteCarloSS::NonScatterEvent) ++nonscatters;
      else if (ae == MonteCarloSS::StartSecondaryEvent) ++secondaries;
   }
};

static void golden_barrier(const std::string& out, SiModel& si)
{
   FILE* f = openw(out, "barrier.txt");
   fprintf(f, "# ExpQMBarrierSM on a vacuum/Si surface: dir(0=Si->vac,1=vac->Si) E theta phi x y z | E' theta' phi' x' y' z' region'(0=vac,1=Si)\n");
   SEmaterialT vacuum;
   ExpQMBarrierSMT vb(&vacuum);
   MONSEL_MaterialScatterModelT vmsm(&vacuum, &vb);
   NullMaterialScatterModelT nullmsm;
   double cen[] = { 0, 0, 0 };
   SphereT sphere(cen, MonteCarloSS::ChamberRadius);
   RegionT chamber(nullptr, &nullmsm, &sphere);
   chamber.updateMaterial(*chamber.getScatterModel(), vmsm);
   NormalMultiPlaneShapeT half;
   double nz[] = { 0., 0., -1. }, o[] = { 0., 0., 0. };
   PlaneT pl(nz, 3, o, 3);
   half.addPlane(pl);
   RegionT siReg(&chamber, si.msm, (NormalShapeT*)&half);
   for (int i = 0; i < 1000; ++i) {
      int dir = i & 1;
      double EeV = (i % 5 == 0) ? 3.75 * (0.5 + uin()) : ::exp(::log(0.5) + (::log(2000.0) - ::log(0.5)) * uin());
      double th = dir ? Math2::PI / 2 * uin() : Math2::PI / 2 + Math2::PI / 2 * uin();
      double ph = 2 * Math2::PI * uin() - Math2::PI;
      double pos[] = { (uin() - 0.5) * 1e-8, (uin() - 0.5) * 1e-8, 0. };
      ElectronT e(pos, th, ph, ToSI::eV(EeV));
      const RegionBaseT* cur = dir ? (RegionBaseT*)&chamber : (RegionBaseT*)&siReg;
      const RegionBaseT* nxt = dir ? (RegionBaseT*)&siReg : (RegionBaseT*)&chamber;
      e.setCurrentRegion(cur);
      // the struck shape's normal is the one the last getFirstNormal call left behind
      double p0[] = { pos[0] - 1e-9 * ::sin(th) * ::cos(ph), pos[1] - 1e-9 * ::sin(th) * ::sin(ph), pos[2] - 1e-9 * ::cos(th) };
      double p1[] = { pos[0] + 1e-9 * ::sin(th) * ::cos(ph), pos[1] + 1e-9 * ::sin(th) * ::sin(ph), pos[2] + 1e-9 * ::cos(th) };
      half.getFirstNormal(p0, p1);
      ((IMaterialScatterModelT*)cur->getScatterModel())->barrierScatter(&e, nxt);
      VectorXd p = e.getPosition();
      fprintf(f, "%d " G " " G " " G " " G " " G " " G " " G " " G " " G " " G " " G " " G " %d\n", dir, ToSI::eV(EeV), th, ph, pos[0], pos[1], pos[2],
         e.getEnergy(), e.getTheta(), e.getPhi(), p[0], p[1], p[2], e.getCurrentRegion() == &siReg ? 1 : 0);
   }
   fclose(f);
}

// ---------------------------------------------------------------- whole runs
static int run_scene(bool lines, int nprim, unsigned long long seed, const std::string& tdir, double beameV,
                     double x0nm, double dxnm, int npix)
{
   g_gen.seed(seed);
   g_queue.clear();
   SiModel si("");
   si.build(tdir);
   PMMAModel pm;
   pm.build();
   SEmaterialT vacuum;
   vacuum.setName("SE vacuum");
   ExpQMBarrierSMT vb(&vacuum);
   MONSEL_MaterialScatterModelT vmsm(&vacuum, &vb);
   NullMaterialScatterModelT nullmsm;
   double cen[] = { 0, 0, 0 };
   SphereT sphere(cen, MonteCarloSS::ChamberRadius);
   double beamE = ToSI::eV(beameV);
   double width = lines ? 1e-9 : 0.0;
   double gunc[] = { 0, 0, -20e-9 };
   GaussianBeamT eg(width, beamE, gunc);
   RegionT chamber(nullptr, &nullmsm, &sphere);
   chamber.updateMaterial(*chamber.getScatterModel(), vmsm);
   NormalMultiPlaneShapeT half;
   double nz[] = { 0., 0., -1. }, o[] = { 0., 0., 0. };
   PlaneT pl(nz, 3, o, 3);
   half.addPlane(pl);
   RegionT siReg(&chamber, si.msm, (NormalShapeT*)&half);
   std::vector<RegionT*> lineRegs;
   double h = 100e-9;
   if (lines) {
      for (int i = 0; i < 3; ++i) {
         NormalIntersectionShapeT* line = make_line(-h, 40e-9, 1e-6, 3 * Math2::PI / 180, 3 * Math2::PI / 180, (i - 1) * 200e-9);
         lineRegs.push_back(new RegionT(&chamber, pm.msm, line));
      }
   }
   MonteCarloSS::MonteCarloSS monte(&eg, &chamber, eg.createElectron());
   int nbins = (int)(beameV / 10.0);
   ScatterCounter cnt;
   monte.addActionListener(cnt);
   auto t0 = std::chrono::steady_clock::now();
   printf("# scene=%s beam_eV=%g nprim=%d seed=%llu nbins=%d\n", lines ? "lines" : "halfspace", beameV, nprim, seed, nbins);
   for (int p = 0; p < npix; ++p) {
      double xnm = x0nm + p * dxnm;
      double c[] = { xnm * 1e-9, 0., lines ? -h - 20e-9 : -20e-9 };
      eg.setCenter(c);
      BackscatterStatsT back(monte, nbins);
      monte.addActionListener(back);
      monte.runMultipleTrajectories(nprim);
      const HistogramT& hist = back.backscatterEnergyHistogram();
      const HistogramT& fwd = back.forwardscatterEnergyHistogram();
      double energyperbineV = beameV / hist.binCount();
      double maxSEbin = 50. / energyperbineV;
      int totalSE = 0;
      for (int j = 0; j < (int)maxSEbin; ++j) totalSE += hist.counts(j);
      double SEf = (float)totalSE / nprim;
      double bsf = back.backscatterFraction() - SEf;
      printf("pixel %g %.17g %.17g %d %d\n", xnm, bsf, SEf, hist.totalCounts(), totalSE);
      printf("back");
      for (int j = -1; j <= hist.binCount(); ++j) printf(" %d", hist.counts(j));
      printf("\nfwd");
      for (int j = -1; j <= fwd.binCount(); ++j) printf(" %d", fwd.counts(j));
      const HistogramT& elev = back.elevationHistogram();
      const HistogramT& azim = back.azimuthalHistogram();
      printf("\nelev");
      for (int j = -1; j <= elev.binCount(); ++j) printf(" %d", elev.counts(j));
      printf("\nazim");
      for (int j = -1; j <= azim.binCount(); ++j) printf(" %d", azim.counts(j));
      printf("\n");
      monte.removeActionListener(back);
   }
   auto t1 = std::chrono::steady_clock::now();
   double secs = std::chrono::duration<double>(t1 - t0).count();
   printf("steps %lld %lld %lld\n", cnt.scatters, cnt.nonscatters, cnt.secondaries);
   printf("seconds %.6f\n", secs);
   return 0;
}

// ---------------------------------------------------------------- rotated shapes
// ITransform::rotate of the Normal shapes that rotate safely (NormalMultiPlaneShape.cu:257-261 through
// MultiPlaneShape::rotate and Plane::rotate, NormalCylindricalShape.cu:324-330), with the Euler-angle
// matrix of Utility/Transform3D.cu (both branches: phi != 0 and the phi == 0 special case).
static void golden_rotate(const std::string& out)
{
   FILE* f = openw(out, "rotate.txt");
   fprintf(f, "# shape(0 block rotated phi,theta,psi about a pivot, 1 block rotated with phi=0, 2 tilted half-space,"
              " 3 cylinder rotated (axis normalised by the rotation), 4 cylinder rotated twice) "
              "p0(3) p1(3) | nx ny nz u contains(p0) contains(p0,p1)\n");
   std::mt19937_64 gin(777);
   auto u = [&]() { return (double)(gin() >> 11) * (1.0 / 9007199254740992.0); };
   auto block = [&]() {
      NormalMultiPlaneShapeT* b = new NormalMultiPlaneShapeT();
      double c[] = { 5e-9, -3e-9, 12e-9 }, h[] = { 15e-9, 10e-9, 5e-9 };
      for (int a = 0; a < 3; ++a)
         for (int sg = -1; sg <= 1; sg += 2) {
            double n[] = { 0, 0, 0 }, p[] = { c[0], c[1], c[2] };
            n[a] = sg;
            p[a] += sg * h[a];
            b->addPlane(*new PlaneT(n, 3, p, 3));
         }
      return b;
   };
   NormalMultiPlaneShapeT* b0 = block();
   const double piv0[] = { 3e-9, -2e-9, 10e-9 };
   b0->rotate(piv0, 0.7, 0.4, -1.1);
   NormalMultiPlaneShapeT* b1 = block();
   const double piv1[] = { -4e-9, 6e-9, 0. };
   b1->rotate(piv1, 0.0, 0.9, 0.3);
   NormalMultiPlaneShapeT* hs = new NormalMultiPlaneShapeT();
   double nz[] = { 0., 0., -1. }, o[] = { 0., 0., 0. };
   hs->addPlane(*new PlaneT(nz, 3, o, 3));
   const double piv2[] = { 10e-9, 0., 0. };
   hs->rotate(piv2, 0.2, 0.3, 0.0);
   double e0[] = { -20e-9, -10e-9, 30e-9 }, e1[] = { 25e-9, 15e-9, 50e-9 };
   NormalCylindricalShapeT* c0 = new NormalCylindricalShapeT(e0, e1, 12e-9);
   const double piv3[] = { 0., 5e-9, 20e-9 };
   c0->rotate(piv3, -0.5, 1.2, 0.8);
   NormalCylindricalShapeT* c1 = new NormalCylindricalShapeT(e0, e1, 9e-9);
   c1->rotate(piv3, 0.0, 0.5, 0.0);
   c1->rotate(piv0, 1.3, -0.2, 0.6);
   NormalShapeT* shapes[] = { (NormalShapeT*)b0, (NormalShapeT*)b1, (NormalShapeT*)hs, (NormalShapeT*)c0,
                              (NormalShapeT*)c1 };
   const double* around[] = { piv0, piv1, piv2, piv3, piv0 };  // segments start near each shape
   for (int s = 0; s < 5; ++s) {
      for (int i = 0; i < 3000; ++i) {
         double p0[3], p1[3];
         for (int k = 0; k < 3; ++k) p0[k] = around[s][k] + (u() * 50 - 25) * 1e-9;
         double len = ::exp(::log(0.05e-9) + (::log(60e-9) - ::log(0.05e-9)) * u());
         double th2 = Math2::PI * u(), ph = 2 * Math2::PI * u();
         p1[0] = p0[0] + len * ::sin(th2) * ::cos(ph);
         p1[1] = p0[1] + len * ::sin(th2) * ::sin(ph);
         p1[2] = p0[2] + len * ::cos(th2);
         VectorXd r = shapes[s]->getFirstNormal(p0, p1);
         int inside = ((ShapeT*)shapes[s])->contains(p0) ? 1 : 0;
         int inside2 = shapes[s]->contains(p0, p1) ? 1 : 0;
         fprintf(f, "%d " G " " G " " G " " G " " G " " G " " G " " G " " G " " G " %d %d\n", s, p0[0], p0[1], p0[2], p1[0],
                 p1[1], p1[2], r[0], r[1], r[2], r[3], inside, inside2);
      }
   }
   fclose(f);
}

// ---------------------------------------------------------------- scene replay
// A scene written by cudamonsel_b200.scenes.SceneSpec.to_text: one construction call per line,
// arguments in SI units, handles = line numbers of earlier calls.  Every call is made on the
// reference's own classes as LinesOnLayers.cu:80-282 makes it.  Calls the reference cannot make
// safely are refused (exit 3): translating or rotating an intersection or union (their casts
// between ITransform and Shape, NormalIntersectionShape.cu:257-263), and a rounded line built
// with the JMONSEL fixes on (the reference always has the left-corner quirk of NShapes.cu:140).
// A line translated before use is assembled at its offset by make_line_at (radius 0 only).
struct RObj {
   int kind = -1;  // 0 material 1 msm 2 table 3 shape 4 region
   SEmaterialT* mat = nullptr;
   MONSEL_MaterialScatterModelT* msm = nullptr;
   std::string path;
   ShapeT* plain = nullptr;     // sphere
   NormalShapeT* ns = nullptr;  // normal shapes
   int skind = 0;               // 1 planes 2 cylinder 3 intersection 4 union 5 line (deferred) 6 sphere
   NormalMultiPlaneShapeT* planes = nullptr;
   NormalCylindricalShapeT* cyl = nullptr;
   double line[7] = { 0, 0, 0, 0, 0, 0, 0 }, off[3] = { 0, 0, 0 };
   bool fixes = false;
   RegionT* region = nullptr;
};

[[noreturn]] static void refuse(const char* what)
{
   fprintf(stderr, "scene not reproducible by the reference: %s\n", what);
   exit(3);
}

// NShapes::createLine (radius 0) with every plane point moved by (dx, dy, dz), as Plane::translate does
static NormalIntersectionShapeT* make_line_at(const double* a, const double* off)
{
   const double topz = a[0], width = a[1], length = a[2], thetal = a[3], thetar = a[4];
   const double dx = off[0], dy = off[1], dz = off[2];
   NormalMultiPlaneShapeT* enclosure = new NormalMultiPlaneShapeT();
   double signz = !topz ? 0 : (topz > 0 ? 1 : -1);
   if (signz == 0.) signz = 1.;
   double n0[] = { 0., 0., signz }, p0[] = { 0. + dx, 0. + dy, topz + dz };
   enclosure->addPlane(*new PlaneT(n0, 3, p0, 3));
   double n1[] = { 0., 0., -signz }, p1[] = { 0. + dx, 0. + dy, 0. + dz };
   enclosure->addPlane(*new PlaneT(n1, 3, p1, 3));
   double n2[] = { 0., 1., 0. }, p2[] = { 0. + dx, length / 2. + dy, 0. + dz };
   enclosure->addPlane(*new PlaneT(n2, 3, p2, 3));
   double n3[] = { 0., -1., 0. }, p3[] = { 0. + dx, -length / 2. + dy, 0. + dz };
   enclosure->addPlane(*new PlaneT(n3, 3, p3, 3));
   NormalMultiPlaneShapeT* rightNMPS = new NormalMultiPlaneShapeT();
   double n4[] = { ::cos(thetar), 0., signz * ::sin(thetar) }, p4[] = { width / 2 + dx, 0. + dy, 0. + dz };
   rightNMPS->addPlane(*new PlaneT(n4, 3, p4, 3));
   NormalMultiPlaneShapeT* leftNMPS = new NormalMultiPlaneShapeT();
   double n6[] = { -::cos(thetal), 0., signz * ::sin(thetal) }, p6[] = { -width / 2 + dx, 0. + dy, 0. + dz };
   leftNMPS->addPlane(*new PlaneT(n6, 3, p6, 3));
   NormalIntersectionShapeT* nts = new NormalIntersectionShapeT(*leftNMPS, *rightNMPS);
   return new NormalIntersectionShapeT(*nts, *enclosure);
}

static NormalShapeT* normal_of(RObj& o)
{
   if (o.kind != 3 || o.skind == 6) refuse("a sphere used as a normal shape");
   if (o.skind == 5 && !o.ns) {
      const bool moved = o.off[0] != 0 || o.off[1] != 0 || o.off[2] != 0;
      if (o.line[5] == 0 && o.line[6] == 0) o.ns = make_line_at(o.line, o.off);
      else if (moved) refuse("a translated rounded line");
      else if (o.fixes) refuse("a rounded line with the JMONSEL fixes");
      else o.ns = NShapes::createLine(o.line[0], o.line[1], o.line[2], o.line[3], o.line[4], o.line[5], o.line[6]);
   }
   return o.ns;
}

static int replay_scene(const char* scenefile, const char* pixfile, unsigned long long seed, double width, bool angles)
{
   std::ifstream in(scenefile);
   if (!in) { perror(scenefile); return 2; }
   std::vector<RObj> ob;
   std::string ln;
   int options = 0, chamber = -1;
   NullMaterialScatterModelT* nullmsm = new NullMaterialScatterModelT();
   while (std::getline(in, ln)) {
      std::istringstream s(ln);
      std::string op;
      s >> op;
      RObj o;
      auto I = [&]() { int v; s >> v; return v; };
      auto D = [&]() { double v; s >> v; return v; };
      if (op == "material") {
         int n = I();
         std::vector<const ElementT*> el(n);
         std::vector<double> A(n), wf(n);
         for (int i = 0; i < n; ++i) el[i] = &Element::byAtomicNumber(I());
         for (int i = 0; i < n; ++i) A[i] = D();
         for (int i = 0; i < n; ++i) wf[i] = D();
         const double density = D(), workfun = D(), ecb = D(), gap = D();
         const int nc = I();
         std::vector<double> core(nc);
         for (int i = 0; i < nc; ++i) core[i] = D();
         o.kind = 0;
         if (n == 0) {
            o.mat = new SEmaterialT();  // vacuum, as LinesOnLayers.cu:80
         } else {
            o.mat = new SEmaterialT(el.data(), n, wf.data(), n, density, (char*)"material");
            o.mat->setWorkfunction(workfun);
            o.mat->setEnergyCBbottom(ecb);
            o.mat->setBandgap(gap);
            if (nc) o.mat->setCoreEnergy(core.data(), nc);
         }
      } else if (op == "msm") {
         SEmaterialT* m = ob[I()].mat;
         o.kind = 1;
         o.mat = m;
         o.msm = new MONSEL_MaterialScatterModelT(m, new ExpQMBarrierSMT(m));
      } else if (op == "table") {
         o.kind = 2;
         s >> o.path;
      } else if (op == "nistmott") {
         RObj& m = ob[I()];
         const int method = I();
         const RandomizedScatterFactoryT& fac = method == 2 ? NISTMottRS::Factory100
                                               : method == 3 ? NISTMottRS::Factory100Lin : NISTMottRS::Factory;
         m.msm->addScatterMechanism(new SelectableElasticSMT(*m.mat, fac));
      } else if (op == "tabulated") {
         RObj& m = ob[I()];
         const int mse = I();
         const double offset = D();
         StringT* t = new StringT[4];
         for (int i = 0; i < 4; ++i) t[i] = ob[I()].path.c_str();
         m.msm->addScatterMechanism(new TabulatedInelasticSMT(*m.mat, mse, t, offset));
      } else if (op == "fitted") {
         RObj& m = ob[I()];
         const double e = D(), b = D();
         m.msm->addScatterMechanism(new FittedInelSMT(*m.mat, e, *new JoyLuoNieminenCSDT(*m.mat, b)));
      } else if (op == "phonon") {
         RObj& m = ob[I()];
         const double a = D(), b = D(), c = D(), d = D(), e = D();
         m.msm->addScatterMechanism(new GanachaudMokraniPhononInelasticSMT(a, b, c, d, e));
      } else if (op == "polaron") {
         RObj& m = ob[I()];
         const double a = D(), b = D();
         m.msm->addScatterMechanism(new GanachaudMokraniPolaronTrapSMT(a, b));
      } else if (op == "csd_jln") {
         RObj& m = ob[I()];
         m.msm->setCSD(new JoyLuoNieminenCSDT(*m.mat, D()));
      } else if (op == "min_e") {
         RObj& m = ob[I()];
         m.msm->setMinEforTracking(D());
      } else if (op == "set_options") {
         options = I();
      } else if (op == "sphere") {
         double c[3] = { D(), D(), D() };
         o.kind = 3;
         o.skind = 6;
         o.plain = new SphereT(c, D());
      } else if (op == "planes") {
         const int n = I();
         std::vector<double> nv(3 * n), pv(3 * n);
         for (auto& x : nv) x = D();
         for (auto& x : pv) x = D();
         o.kind = 3;
         o.skind = 1;
         o.planes = new NormalMultiPlaneShapeT();
         for (int i = 0; i < n; ++i) o.planes->addPlane(*new PlaneT(&nv[3 * i], 3, &pv[3 * i], 3));
         o.ns = (NormalShapeT*)o.planes;
      } else if (op == "cylinder") {
         double e0[3] = { D(), D(), D() }, e1[3] = { D(), D(), D() };
         o.kind = 3;
         o.skind = 2;
         o.cyl = new NormalCylindricalShapeT(e0, e1, D());
         if (options & 1) {  // the axis normalised: an identity rotation recomputes it from the set length
            const double zero[] = { 0., 0., 0. };
            o.cyl->rotate(zero, 0., 0., 0.);
         }
         o.ns = (NormalShapeT*)o.cyl;
      } else if (op == "intersection" || op == "union") {
         NormalShapeT* a = normal_of(ob[I()]);
         NormalShapeT* b = normal_of(ob[I()]);
         o.kind = 3;
         o.skind = op == "union" ? 4 : 3;
         if (op == "union") o.ns = new NormalUnionShapeT(*a, *b);
         else o.ns = new NormalIntersectionShapeT(*a, *b);
      } else if (op == "line") {
         o.kind = 3;
         o.skind = 5;
         for (int i = 0; i < 7; ++i) o.line[i] = D();
         o.fixes = (options & 1) != 0;
      } else if (op == "translate") {
         RObj& t = ob[I()];
         double d[3] = { D(), D(), D() };
         if (t.skind == 5 && !t.ns) for (int i = 0; i < 3; ++i) t.off[i] += d[i];
         else if (t.skind == 1) t.planes->translate(d);
         else if (t.skind == 2) t.cyl->translate(d);
         else refuse("translating a composite shape");
      } else if (op == "rotate") {
         RObj& t = ob[I()];
         double pv[3] = { D(), D(), D() };
         const double phi = D(), th = D(), psi = D();
         if (t.skind == 1) t.planes->rotate(pv, phi, th, psi);
         else if (t.skind == 2) t.cyl->rotate(pv, phi, th, psi);
         else refuse("rotating a composite shape");
      } else if (op == "region") {
         const int parent = I(), m = I(), sh = I();
         o.kind = 4;
         ShapeT* shape = ob[sh].skind == 6 ? ob[sh].plain : (ShapeT*)normal_of(ob[sh]);
         if (parent < 0) {  // the chamber: a null model replaced by the vacuum's (LinesOnLayers.cu:80-84)
            o.region = new RegionT(nullptr, nullmsm, shape);
            o.region->updateMaterial(*o.region->getScatterModel(), *ob[m].msm);
            chamber = (int)ob.size();
         } else {
            o.region = new RegionT(ob[parent].region, ob[m].msm, shape);
         }
      } else if (!op.empty()) {
         fprintf(stderr, "unknown scene call %s\n", op.c_str());
         return 2;
      }
      ob.push_back(o);
   }
   if (options) refuse("a run with the JMONSEL fixes on");
   if (chamber < 0) { fprintf(stderr, "no chamber\n"); return 2; }
   std::ifstream pin(pixfile);
   if (!pin) { perror(pixfile); return 2; }
   struct Px { double c[3], E; int n, nb; };
   std::vector<Px> px;
   Px p;
   while (pin >> p.c[0] >> p.c[1] >> p.c[2] >> p.E >> p.n >> p.nb) px.push_back(p);
   g_gen.seed(seed);
   g_queue.clear();
   double gunc[] = { 0, 0, -20e-9 };
   GaussianBeamT eg(width, px.empty() ? ToSI::eV(500.) : px[0].E, gunc);
   MonteCarloSS::MonteCarloSS monte(&eg, ob[chamber].region, eg.createElectron());
   ScatterCounter cnt;
   monte.addActionListener(cnt);
   auto t0 = std::chrono::steady_clock::now();
   printf("# scene=%s pixels=%zu seed=%llu width=%g\n", scenefile, px.size(), seed, width);
   for (const Px& q : px) {
      eg.setCenter(q.c);
      eg.setBeamEnergy(q.E);
      BackscatterStatsT back(monte, q.nb);
      monte.addActionListener(back);
      monte.runMultipleTrajectories(q.n);
      const HistogramT& hist = back.backscatterEnergyHistogram();
      const HistogramT& fwd = back.forwardscatterEnergyHistogram();
      printf("pixel %.17g %.17g %.17g %d\nback", q.c[0], q.c[1], q.c[2], q.n);
      for (int j = -1; j <= hist.binCount(); ++j) printf(" %d", hist.counts(j));
      printf("\nfwd");
      for (int j = -1; j <= fwd.binCount(); ++j) printf(" %d", fwd.counts(j));
      printf("\n");
      if (angles) {
         const HistogramT& elev = back.elevationHistogram();
         const HistogramT& azim = back.azimuthalHistogram();
         printf("elev");
         for (int j = -1; j <= elev.binCount(); ++j) printf(" %d", elev.counts(j));
         printf("\nazim");
         for (int j = -1; j <= azim.binCount(); ++j) printf(" %d", azim.counts(j));
         printf("\n");
      }
      monte.removeActionListener(back);
   }
   auto t1 = std::chrono::steady_clock::now();
   printf("steps %lld %lld %lld\n", cnt.scatters, cnt.nonscatters, cnt.secondaries);
   printf("seconds %.6f\n", std::chrono::duration<double>(t1 - t0).count());
   return 0;
}

int main(int argc, char** argv)
{
   if (argc < 2) {
      fprintf(stderr, "usage: ref_driver golden <outdir> <SiTablesDir> | run1 <nprim> <seed> <SiTablesDir> [beam_eV] | run2 ...\n");
      return 2;
   }
   std::string mode = argv[1];
   // silence the reference's chatty loaders
   FILE* keep = stdout;
   stdout = fopen("/dev/null", "w");
   init_reference();
   fclose(stdout);
   stdout = keep;
   if (mode == "golden" && argc >= 4) {
      std::string out = argv[2];
      SiModel si("");
      si.build(argv[3]);
      PMMAModel pm;
      pm.build();
      golden_nistmott(out);
      golden_nutable(out, si);
      golden_tabinel(out, si);
      golden_elastic(out, si, pm);
      golden_pmma(out, pm);
      golden_phonon(out);
      golden_shapes(out);
      golden_misc(out, si);
      golden_barrier(out, si);
      golden_shapes2(out);
      golden_nistmott23(out);  // last, so the earlier sets keep their input streams
      return 0;
   }
   if (mode == "golden2" && argc >= 3) {  // sets added later, each with its own input stream
      golden_rotate(argv[2]);
      return 0;
   }
   if (mode == "run1" && argc >= 5) {
      double E = argc > 5 ? atof(argv[5]) : 1000.0;
      return run_scene(false, atoi(argv[2]), strtoull(argv[3], 0, 10), argv[4], E, 0.0, 0.0, 1);
   }
   if (mode == "run2" && argc >= 8) {
      double E = argc > 8 ? atof(argv[8]) : 500.0;
      return run_scene(true, atoi(argv[2]), strtoull(argv[3], 0, 10), argv[4], E, atof(argv[5]), atof(argv[6]), atoi(argv[7]));
   }
   if (mode == "scene" && argc >= 6) {
      const bool angles = argc > 6 && std::string(argv[6]) == "angles";
      return replay_scene(argv[2], argv[3], strtoull(argv[4], 0, 10), atof(argv[5]), angles);
   }
   fprintf(stderr, "bad arguments\n");
   return 2;
}
