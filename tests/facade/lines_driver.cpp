// A LinesOnLayers-style driver (the shape of JMONSELTests/LinesOnLayers.cu:37-399) written against the
// reference's C++ API and compiled against include/cudamonsel_b200.hpp: PMMA trapezoid lines on a Si
// substrate, a Gaussian beam scanned across the middle line, BackscatterStats per landing point.  The
// scene is the one tests/test_gpu_facade.py builds through the C ABI (cudamonsel_b200.scenes.lines), so
// the same seeds give the same tallies both ways.
//
//   lines_driver <SiTablesDir> <npix> <ntraj> <seed> [fp64]
// prints one row per pixel: "pixel x_nm BSE SE" and "back c(-1) .. c(nbins)".
#include <cstdio>
#include <cstdlib>
#include <string>

#include "cudamonsel_b200.hpp"

int main(int argc, char** argv)
{
   if (argc < 5) {
      fprintf(stderr, "usage: lines_driver <SiTablesDir> <npix> <ntraj> <seed> [fp64]\n");
      return 2;
   }
   const std::string tableDir = argv[1];
   const int npix = atoi(argv[2]), nTrajectories = atoi(argv[3]);
   cudamonsel::set_seed(strtoull(argv[4], nullptr, 10));
   if (argc > 5 && std::string(argv[5]) == "fp64") cudamonsel::set_precision(CM_PREC_FP64);

   const double meterspernm = 1.e-9;
   const double beamEeV = 500., beamsizenm = 1.;
   const int nlines = 3;
   const double pitchnm = 200., hnm = 100., wnm = 40., linelengthnm = 1000., thetadeg = 3.;

   SEmaterialT vacuum;
   vacuum.setName("SE vacuum");
   ExpQMBarrierSMT vacuumBarrier(&vacuum);
   MONSEL_MaterialScatterModelT vacuumMSM(&vacuum, &vacuumBarrier);

   // PMMA
   const double breakE = ToSI::eV(45.), workfunPMMA = 5.5, bandgapPMMA = 5.;
   const ElementT* componentsCOH[] = { &Element::C, &Element::O, &Element::H };
   const double compositionCOH[] = { 5, 2, 8 };
   CompositionT PMMAcomp;
   PMMAcomp.defineByMoleFraction(componentsCOH, 3, compositionCOH, 3);
   SEmaterialT PMMA(PMMAcomp, 1190.);
   PMMA.setName("PMMA");
   PMMA.setWorkfunction(ToSI::eV(workfunPMMA));
   PMMA.setBandgap(ToSI::eV(bandgapPMMA));
   PMMA.setEnergyCBbottom(ToSI::eV(-workfunPMMA + bandgapPMMA));
   SelectableElasticSMT PMMANISTMott(PMMA, NISTMottRS::Factory);
   JoyLuoNieminenCSDT PMMACSD(PMMA, breakE);
   FittedInelSMT PMMAfittedInel(PMMA, ToSI::eV(65.4), PMMACSD);
   GanachaudMokraniPolaronTrapSMT PMMApolaron(2.e7, 1. / ToSI::eV(4.));
   ExpQMBarrierSMT pmmaBarrier(&PMMA);
   MONSEL_MaterialScatterModelT PMMAMSM(&PMMA, &pmmaBarrier);
   PMMAMSM.addScatterMechanism(&PMMANISTMott);
   PMMAMSM.addScatterMechanism(&PMMAfittedInel);
   PMMAMSM.addScatterMechanism(&PMMApolaron);
   PMMAMSM.setCSD(&PMMACSD);

   // Si
   const double workfunSi = 4.85, bandgapSi = 1.1;
   const ElementT* componentsSi[] = { &Element::Si };
   const double compositionSi[] = { 1. };
   SEmaterialT Si(componentsSi, 1, compositionSi, 1, 2330., "Silicon");
   Si.setWorkfunction(ToSI::eV(workfunSi));
   Si.setEnergyCBbottom(ToSI::eV(-workfunSi + bandgapSi));
   Si.setBandgap(ToSI::eV(bandgapSi));
   const double core[] = { ToSI::eV(99.2), ToSI::eV(99.8), ToSI::eV(149.7), ToSI::eV(1839.) };
   Si.setCoreEnergy(core, 4);
   StringT tables[] = { tableDir + "/IIMFPFullPennInterpSiSI.csv", tableDir + "/interpNUSimReducedDeltaEFullPennSiSI.csv",
                        tableDir + "/interpNUThetaFullPennSiBGSI.csv", tableDir + "/interpSimESE0NUSiBGSI.csv" };
   SelectableElasticSMT SiNISTMott(Si, NISTMottRS::Factory);
   TabulatedInelasticSMT SiInelastic(Si, 3, tables, ToSI::eV(13.54));
   ExpQMBarrierSMT siBarrier(&Si);
   MONSEL_MaterialScatterModelT SiMSM(&Si, &siBarrier);
   SiMSM.addScatterMechanism(&SiNISTMott);
   SiMSM.addScatterMechanism(&SiInelastic);

   // geometry: the chamber, the substrate (material at z >= 0), the lines above it
   const double center[] = { 0., 0., 0. };
   SphereT sphere(center, MonteCarloSS::MonteCarloSS::ChamberRadius);
   NullMaterialScatterModelT NULL_MSM;
   RegionT chamber(nullptr, &NULL_MSM, &sphere);
   chamber.updateMaterial(*chamber.getScatterModel(), vacuumMSM);
   const double normalvector[] = { 0., 0., -1. }, origin[] = { 0., 0., 0. };
   NormalMultiPlaneShapeT substrate;
   PlaneT pl(normalvector, 3, origin, 3);
   substrate.addPlane(pl);
   RegionT substrateRegion(&chamber, &SiMSM, (NormalShapeT*)&substrate);
   const double theta = thetadeg * Math2::PI / 180.;
   for (int i = 0; i < nlines; ++i) {
      NormalIntersectionShapeT* line = (NormalIntersectionShapeT*)NShapes::createLine(
         -hnm * meterspernm, wnm * meterspernm, linelengthnm * meterspernm, theta, theta, 0., 0.);
      const double pos[] = { (i - (nlines - 1) / 2.) * pitchnm * meterspernm, 0., 0. };
      line->translate(pos);
      new RegionT(&chamber, &PMMAMSM, line);  // a region lives as long as the chamber, as in the reference
   }

   const double egCenter[] = { 0., 0., -hnm * meterspernm - 20. * meterspernm };
   GaussianBeamT eg(beamsizenm * meterspernm, ToSI::eV(beamEeV), egCenter);
   MonteCarloSS::MonteCarloSS monte(&eg, &chamber, eg.createElectron());
   const int nbins = (int)(beamEeV / 10.);
   for (int p = 0; p < npix; ++p) {
      const double xnm = (p - (npix - 1) / 2.) * 1.0;
      const double c[] = { xnm * meterspernm, 0., -hnm * meterspernm - 20. * meterspernm };
      eg.setCenter(c);
      BackscatterStatsT back(monte, nbins);
      monte.addActionListener(back);
      monte.runMultipleTrajectories(nTrajectories);
      const HistogramT& hist = back.backscatterEnergyHistogram();
      const double energyperbineV = beamEeV / hist.binCount();
      const double maxSEbin = 50. / energyperbineV;
      int totalSE = 0;
      for (int j = 0; j < (int)maxSEbin; ++j) totalSE += hist.counts(j);
      const double SEf = (float)totalSE / nTrajectories;
      const double bsf = back.backscatterFraction() - SEf;
      printf("pixel %.3f %.9f %.9f\nback", xnm, bsf, SEf);
      for (int j = -1; j <= hist.binCount(); ++j) printf(" %d", hist.counts(j));
      printf("\n");
      monte.removeActionListener(back);
   }
   return 0;
}
