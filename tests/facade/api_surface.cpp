// The rest of the reference's API the facade keeps (include/cudamonsel_b200.hpp), in a small scene: Si with
// the phonon mechanism, a PMMA block rotated about a pivot, a cylinder, a union, a rounded createLine, a
// deep-Si model with its own tracking cut and a tunnelling barrier, and every BackscatterStats histogram.
//
//   api_surface [fp64]      runs 200 trajectories at one landing point and prints the tallies
#include <cstdio>
#include <string>

#include "cudamonsel_b200.hpp"

int main(int argc, char** argv)
{
   if (argc > 1 && std::string(argv[1]) == "fp64") cudamonsel::set_precision(CM_PREC_FP64);
   cudamonsel::set_seed(7);
   const double nm = 1.e-9;

   SEmaterialT vacuum;
   ExpQMBarrierSMT vacuumBarrier(&vacuum);
   MONSEL_MaterialScatterModelT vacuumMSM(&vacuum, &vacuumBarrier);

   const ElementT* si[] = { &Element::byAtomicNumber(14) };
   const double one[] = { 1. };
   SEmaterialT Si(si, 1, one, 1, 2330., "Silicon");
   Si.setWorkfunction(ToSI::eV(4.85));
   Si.setEnergyCBbottom(ToSI::eV(-3.75));
   Si.setBandgap(ToSI::eV(1.1));
   Si.addCoreEnergy(ToSI::eV(99.2));
   Si.addCoreEnergy(ToSI::eV(149.7));
   const std::string dir = std::string(cm_data_dir()) + "/ScatteringTables/SiTables";
   StringT tables[] = { dir + "/IIMFPFullPennInterpSiSI.csv", dir + "/interpNUSimReducedDeltaEFullPennSiSI.csv",
                        dir + "/interpNUThetaFullPennSiBGSI.csv", dir + "/interpSimESE0NUSiBGSI.csv" };
   SelectableElasticSMT SiMott(Si, NISTMottRS::Factory100Lin);
   TabulatedInelasticSMT SiInel(Si, 3, tables, ToSI::eV(13.54));
   GanachaudMokraniPhononInelasticSMT SiPhonon(3., ToSI::eV(0.063), 300., 11.7, 1.);
   ExpQMBarrierSMT SiBarrier(&Si, 1.e-9);  // tunnelling barrier with a 1 nm length scale
   MONSEL_MaterialScatterModelT SiMSM(&Si, &SiBarrier);
   SiMSM.addScatterMechanism(&SiMott);
   SiMSM.addScatterMechanism(&SiInel);
   SiMSM.addScatterMechanism(&SiPhonon);
   MONSEL_MaterialScatterModelT SiMSMDeep = SiMSM;  // a copy with its own tracking cut
   SiMSMDeep.setMinEforTracking(ToSI::eV(50.));

   const ElementT* coh[] = { &Element::C, &Element::O, &Element::H };
   const double moles[] = { 5, 2, 8 };
   CompositionT comp;
   comp.defineByMoleFraction(coh, 3, moles, 3);
   SEmaterialT PMMA(comp, 1190.);
   PMMA.setWorkfunction(ToSI::eV(5.5));
   PMMA.setBandgap(ToSI::eV(5.));
   PMMA.setEnergyCBbottom(ToSI::eV(-0.5));
   SelectableElasticSMT PMMAMott(PMMA, NISTMottRS::Factory);
   JoyLuoNieminenCSDT csd(PMMA, ToSI::eV(45.));
   FittedInelSMT fitted(PMMA, ToSI::eV(65.4), csd);
   GanachaudMokraniPolaronTrapSMT polaron(2.e7, 1. / ToSI::eV(4.));
   ExpQMBarrierSMT PMMABarrier(&PMMA);
   MONSEL_MaterialScatterModelT PMMAMSM(&PMMA, &PMMABarrier);
   PMMAMSM.addScatterMechanism(&PMMAMott);
   PMMAMSM.addScatterMechanism(&fitted);
   PMMAMSM.addScatterMechanism(&polaron);
   PMMAMSM.setCSD(&csd);

   const double origin[] = { 0., 0., 0. };
   SphereT sphere(origin, MonteCarloSS::MonteCarloSS::ChamberRadius);
   RegionT chamber(nullptr, &vacuumMSM, &sphere);
   const double nz[] = { 0., 0., -1. };
   NormalMultiPlaneShapeT substrate;
   substrate.addPlane(PlaneT(nz, 3, origin, 3));
   RegionT substrateRegion(&chamber, &SiMSM, (NormalShapeT*)&substrate);
   const double deepPos[] = { 0., 0., 300. * nm };
   NormalMultiPlaneShapeT deep;
   deep.addPlane(PlaneT(nz, 3, deepPos, 3));
   RegionT deepRegion(&substrateRegion, &SiMSMDeep, (NormalShapeT*)&deep);

   NormalMultiPlaneShapeT block;  // 40 x 40 x 30 nm PMMA block, then turned 20 deg about z around its centre
   const double c[] = { 60. * nm, 0., -15. * nm }, h[] = { 20. * nm, 20. * nm, 15. * nm };
   for (int a = 0; a < 3; ++a)
      for (int sg = -1; sg <= 1; sg += 2) {
         double n[] = { 0., 0., 0. }, p[] = { c[0], c[1], c[2] };
         n[a] = sg;
         p[a] += sg * h[a];
         block.addPlane(n, p);
      }
   block.rotate(c, 20. * Math2::PI / 180., 0., 0.);
   RegionT blockRegion(&chamber, &PMMAMSM, (NormalShapeT*)&block);

   cudamonsel::set_options(CM_OPT_JMONSEL_FIXES);  // shapes built now take the JMONSEL fixes (see the header)
   const double e0[] = { -60. * nm, -200. * nm, -25. * nm }, e1[] = { -60. * nm, 200. * nm, -25. * nm };
   NormalCylindricalShapeT cyl(e0, e1, 25. * nm);
   NormalMultiPlaneShapeT cap;
   const double up[] = { 0., 0., 1. }, capPos[] = { 0., 0., -10. * nm };
   cap.addPlane(up, capPos);
   NormalIntersectionShapeT capped(cyl, cap);
   const double b0[] = { -150. * nm, -200. * nm, -20. * nm }, b1[] = { -150. * nm, 200. * nm, -20. * nm };
   NormalCylindricalShapeT cyl2(b0, b1, 20. * nm);
   NormalUnionShapeT both(capped, cyl2);
   RegionT featureRegion(&chamber, &PMMAMSM, &both);
   NormalShapeT* line = NShapes::createLine(-60. * nm, 40. * nm, 400. * nm, 0.05, 0.05, 8. * nm, 8. * nm);
   const double shift[] = { 150. * nm, 0., 0. };
   line->translate(shift);
   RegionT lineRegion(&chamber, &PMMAMSM, line);
   cudamonsel::set_options(0);

   const double gun[] = { 60. * nm, 0., -60. * nm };
   GaussianBeamT eg(2. * nm, ToSI::eV(800.), gun);
   MonteCarloSS::MonteCarloSS monte(&eg, &chamber, eg.createElectron());
   BackscatterStatsT back(monte, 80);
   monte.addActionListener(back);
   monte.runMultipleTrajectories(200);
   monte.removeActionListener(back);
   const HistogramT& b = back.backscatterEnergyHistogram();
   const HistogramT& f = back.forwardscatterEnergyHistogram();
   printf("bins %d back %d fwd %d elevation %d azimuth %d fractions %.6f %.6f %.6f edges %.3f %.3f\n",
          b.binCount(), b.totalCounts(), f.totalCounts(), back.elevationHistogram().totalCounts(),
          back.azimuthalHistogram().totalCounts(), back.backscatterFraction(), back.forwardscatterFraction(),
          back.scatterFraction(), b.minValue(0), b.maxValue(b.binCount() - 1));
   return 0;
}
