// vhlle_run -- the reference driver's evolution loop (src/main.cpp:273-441)
// over the device hydro: parameters file, substeps, one-shot x2 resize,
// termination at tauMax.  The initial state (src/main.cpp:320-366) is built
// on the device by the reference's modules for icModel 2 (IC over the s95p
// table of -ISinput, s0ScaleFactor, glauberVar), 3 (IcPartUrqmd, the
// particle list of -ISinput smeared with Rgt, Rgz), 4 (ICGubser), 5
// (IcGlissando) and 7 (IcTrento), the last two reading -ISinput with the
// setup named by -system, at tau0; or, whatever icModel says, it is read
// from -ISinput when that file is a grid snapshot (VHBSNAP1, which fixes
// tau0).  The other models (the GSL optical Glauber, the SMASH particle
// lists, TRENTO 3D, SuperMC) are refused.
//
//   vhlle_run -params FILE [-ISinput SNAPSHOT|ICFILE] [-outputDir DIR]
//             [-system S] [-printParams]
//
// Parameters are read exactly as the reference reads them (same keys,
// defaults, "CCC"/"UUU" echo).  The hydro EoS is the EoS1f table named by
// the extra key eos1fFile; else, for eosType 1 (the default), EoSChiral from
// ./eos/chiraleos.dat and ./eos/chiralsmall.dat as the reference reads them;
// for eosType 2, EoSAZH from ./eos/azhydro0p2; for eosType 4, EoSCMFe from
// ./eos/cmfe.dat and ./eos/cmfe_small.dat;
// else (those files absent, or another eosType) the conformal gas of 47.5
// degrees of freedom.  The freeze-out EoS (src/main.cpp:304-314) is, for
// eosTypeHadron 0, EoSHadron from ./eos/eosHadronLog.dat, for eosTypeHadron
// 1, EoSSmash from ./eos/hadgas_eos_SMASH.dat (101 x 51 x 51), where those
// files exist; otherwise the hydro EoS.  Before the loop the corona of Fluid::outputCorona opens the
// freeze-out file.  Each loop iteration does what Fluid::outputSurface does: it
// appends the freeze-out elements to DIR/freezeout.dat.unfinished (renamed
// freezeout.dat at the end) and prints the same line (tau, E, Efull,
// nbSurf, S, EtotSurf, elements, suspicious elements, cut-cell fraction);
// the loop stops at tauMax or when an iteration finds no element, as the
// reference's does.  With the key vorticity set, DIR/beta.dat gets the
// header after the corona and each iteration's beta.dat lines.  The final
// grid is written to DIR/final.vhb.
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>

#include "vhlle_b200.hpp"

namespace {

struct CommandLine {
  std::string collSystem, isInputFile, outputDir = "data", params;
  bool printParams = false;
};

// readCommandLine, src/main.cpp:226-243 (same flags, value after the flag)
CommandLine readCommandLine(int argc, char** argv, vhb::Params& P) {
  CommandLine c;
  if (argc == 1) throw vhb::Error(VH_ERR_ARG, "no CL params - exiting.");
  for (int i = 1; i < argc; i++)
    if (std::strcmp(argv[i], "-printParams") == 0) c.printParams = true;
  for (int i = 1; i < argc - 1; i++) {
    if (std::strcmp(argv[i], "-system") == 0) c.collSystem = argv[i + 1];
    if (std::strcmp(argv[i], "-params") == 0) {
      c.params = argv[i + 1];
      std::cout << "vhlle: reading parameters from " << c.params << std::endl;
      P.read(argv[i + 1], std::cout);
    }
    if (std::strcmp(argv[i], "-ISinput") == 0) c.isInputFile = argv[i + 1];
    if (std::strcmp(argv[i], "-outputDir") == 0) c.outputDir = argv[i + 1];
  }
  P.outputDir = c.outputDir;
  P.isInputFile = c.isInputFile;
  P.collSystem = c.collSystem;
  return c;
}

void printParameters(const vhb::Params& P) {
  std::cout << std::setprecision(17);
  std::cout << "====== parameters ======\n"
            << "outputDir = " << P.outputDir << "\n"
            << "eos1fFile = " << P.eos1fFile << "\n"
            << "nx = " << P.nx << "\nny = " << P.ny << "\nnz = " << P.nz << "\n"
            << "xmin = " << P.xmin << "\nxmax = " << P.xmax << "\n"
            << "ymin = " << P.ymin << "\nymax = " << P.ymax << "\n"
            << "etamin = " << P.etamin << "\netamax = " << P.etamax << "\n"
            << "tau0 = " << P.tau0 << "\ntauMax = " << P.tauMax << "\n"
            << "tauGridResize = " << P.tauResize << "\ndtau = " << P.dtau << "\n"
            << "e_crit = " << P.eCrit << "\n"
            << "zetaSparam = " << P.zetaSparam << "\netaSparam = " << P.etaSparam << "\n"
            << "etaS = " << P.etaS << "\nzetaS = " << P.zetaS << "\n"
            << "al = " << P.al << "\nah = " << P.ah << "\naRho = " << P.aRho << "\n"
            << "T0 = " << P.T0 << "\netaSMin = " << P.etaSMin << "\n"
            << "etaSEpsilonMin = " << P.etaSEpsilonMin << "\n"
            << "etaSShiftMuB = " << P.etaSShiftMuB << "\netaSScaleMuB = " << P.etaSScaleMuB
            << "\n"
            << "zetaSPeakEpsilon = " << P.zetaSPeakEpsilon << "\n"
            << "zetaSScaleBeta = " << P.zetaSScaleBeta << "\n"
            << "zetaSSigmaMinus = " << P.zetaSSigmaMinus << "\n"
            << "zetaSSigmaPlus = " << P.zetaSSigmaPlus << "\n"
            << "VTK_output_values = " << P.vtk_values << "\n"
            << "======= end parameters =======" << std::endl;
}

int run(int argc, char** argv) {
  vhb::Params P;
  const CommandLine cl = readCommandLine(argc, argv, P);
  printParameters(P);
  if (cl.printParams) return 0;
  bool snapshot = false;
  if (!cl.isInputFile.empty()) {
    std::ifstream in(cl.isInputFile, std::ios::binary);
    char tag[8] = {};
    in.read(tag, 8);
    snapshot = in && std::memcmp(tag, "VHBSNAP1", 8) == 0;
  }
  if (!snapshot && P.icModel != 2 && P.icModel != 3 && P.icModel != 4 && P.icModel != 5 &&
      P.icModel != 7)
    throw vhb::Error(VH_ERR_ARG, "icModel " + std::to_string(P.icModel) +
                                     " is not built here: give a grid snapshot as -ISinput");
  if (!snapshot && P.icModel != 4 && cl.isInputFile.empty())
    throw vhb::Error(VH_ERR_ARG, "no -ISinput given");

  const double hbarc = 0.1973269804, deg = 16.0 + 3.0 * 12.0 * (7.0 / 8.0);
  struct stat sb;
  const bool chiral = P.eos1fFile.empty() && P.eosType == 1 &&
                      stat("eos/chiraleos.dat", &sb) == 0 && stat("eos/chiralsmall.dat", &sb) == 0;
  const bool azh = P.eos1fFile.empty() && P.eosType == 2 &&
                   stat("eos/azhydro0p2/aa1_p.dat", &sb) == 0;
  const bool cmfe = P.eos1fFile.empty() && P.eosType == 4 && stat("eos/cmfe.dat", &sb) == 0 &&
                    stat("eos/cmfe_small.dat", &sb) == 0;
  vhb::EoS* eos;
  if (!P.eos1fFile.empty())
    eos = new vhb::EoS1f(P.eos1fFile.c_str());
  else if (chiral)  // src/main.cpp:291-292, the tables under ./eos as there
    eos = new vhb::EoSChiral(".");
  else if (azh)  // src/main.cpp:293-294
    eos = new vhb::EoSAZH(".");
  else if (cmfe)  // src/main.cpp:297-298
    eos = new vhb::EoSCMFe(".");
  else
    eos = new vhb::EoSConformal(3.0 * deg * M_PI * M_PI / 90.0 / (hbarc * hbarc * hbarc));
  std::cout << "hydro EoS: "
            << (!P.eos1fFile.empty() ? "EoS1f " + P.eos1fFile
                : chiral ? std::string("EoSChiral (eos/chiraleos.dat, eos/chiralsmall.dat)")
                : azh    ? std::string("EoSAZH (eos/azhydro0p2)")
                : cmfe   ? std::string("EoSCMFe (eos/cmfe.dat, eos/cmfe_small.dat)")
                         : std::string("conformal gas"))
            << std::endl;
  vhb::EoS* eosH = eos;
  if (P.eosTypeHadron == 0 && stat("eos/eosHadronLog.dat", &sb) == 0)
    eosH = new vhb::EoSHadron("eos/eosHadronLog.dat");
  else if (P.eosTypeHadron == 1 && stat("eos/hadgas_eos_SMASH.dat", &sb) == 0)
    eosH = new vhb::EoSSmash("eos/hadgas_eos_SMASH.dat", 101, 51, 51);
  else if (P.eosTypeHadron != 0 && P.eosTypeHadron != 1) {  // src/main.cpp:310-314
    std::cout << "Unknown hadronic EoS type for hypersurface creation.\n"
              << "eosTypeHadron should be either \"0\" (PDG hadronic EoS) or \"1\" (SMASH "
                 "hadronic EoS).\n";
    delete eos;
    return 0;
  }
  std::cout << "freeze-out EoS: "
            << (eosH == eos ? std::string("the hydro EoS")
                            : P.eosTypeHadron == 0 ? std::string("EoSHadron (eos/eosHadronLog.dat)")
                                                   : std::string("EoSSmash (eos/hadgas_eos_SMASH.dat)"))
            << std::endl;
  vhb::TransportCoeff* trcoeff = new vhb::TransportCoeff(
      P.etaS, P.zetaS, P.ah, P.al, P.aRho, P.T0, P.etaSMin, P.etaSEpsilonMin, P.etaSShiftMuB,
      P.etaSScaleMuB, P.zetaSPeakEpsilon, P.zetaSScaleBeta, P.zetaSSigmaMinus,
      P.zetaSSigmaPlus, eos, P.etaSparam, P.zetaSparam);

  vhb::Fluid* f = new vhb::Fluid(eos, eosH, trcoeff, P.nx, P.ny, P.nz, P.xmin, P.xmax, P.ymin,
                                 P.ymax, P.etamin, P.etamax, P.dtau, P.eCrit);
  double tau0 = P.tau0;
  if (snapshot) {
    const auto hdr = vhb::Fluid::readSnapshotHeader(cl.isInputFile.c_str());
    if (hdr.grid.nx != P.nx || hdr.grid.ny != P.ny || hdr.grid.nz != P.nz ||
        hdr.grid.xmin != P.xmin || hdr.grid.xmax != P.xmax || hdr.grid.ymin != P.ymin ||
        hdr.grid.ymax != P.ymax || hdr.grid.etamin != P.etamin || hdr.grid.etamax != P.etamax)
      throw vhb::Error(VH_ERR_ARG, "the snapshot's grid differs from the parameters' grid");
    f->loadSnapshot(cl.isInputFile.c_str());
    tau0 = hdr.tau;  // the snapshot fixes the start time
  }
  std::cout << "fluid allocation done\n";

  vhb::Hydro* h = new vhb::Hydro(f, eos, trcoeff, tau0, P.dtau);
  if (!snapshot) {  // src/main.cpp:324-366, the modules built on the device
    const char* file = cl.isInputFile.c_str();
    const char* sys = cl.collSystem.c_str();
    if (P.icModel == 2) {
      vhb::IC(file, P.s0ScaleFactor, P.glauberVariable).setIC(h);
    } else if (P.icModel == 3) {
      vhb::IcPartUrqmd ic(f, file, P.Rgt, P.Rgz, tau0);
      ic.setIC(h);
      std::cout << "IcPartUrqmd: loaded " << ic.nevents() << " events\n";
    } else if (P.icModel == 4) {
      vhb::ICGubser().setIC(h);
    } else if (P.icModel == 5) {
      vhb::IcGlissando ic(f, file, tau0, sys);
      const auto n = ic.setIC(h);
      std::cout << "IcGlissando: loaded " << ic.nevents() << " events, sNorm set to " << n.first
                << "\n";
    } else {
      vhb::IcTrento ic(f, file, tau0, sys);
      const auto n = ic.setIC(h);
      std::cout << "IcTrento: loaded " << ic.nevents() << " events, sNorm set to " << n.first
                << "\n";
    }
  }
  std::cout << "IC done (tau0 = " << tau0 << ")\n";
  if (P.vorticityOn) h->enableVorticity();  // src/main.cpp:379-382
  // Fluid::initOutput (src/fld.cpp:119-129): the output directory and a
  // fresh freezeout.dat.unfinished
  mkdir(cl.outputDir.c_str(), 0755);
  const std::string fo = cl.outputDir + "/freezeout.dat";
  const std::string fo_unf = fo + ".unfinished";
  std::remove(fo.c_str());
  std::remove(fo_unf.c_str());
  const std::string beta = cl.outputDir + "/beta.dat";  // src/fld.cpp:131-136
  if (P.vorticityOn) std::remove(beta.c_str());
  bool resized = false;
  int nloops = 0;
  long nelements = 0;
  std::cout << std::setprecision(6);
  {
    // Fluid::outputCorona at tau0 (src/main.cpp:390, src/fld.cpp:876-1089):
    // the corona elements go first into the freeze-out file; the lines it
    // prints (src/fld.cpp:1075-1088)
    const vh_surface_info ci = h->corona();
    h->writeSurface(fo_unf.c_str(), P.freezeoutExtend);
    const vhb::Totals t = h->totals();
    std::cout << std::setw(10) << "tau" << std::setw(13) << "E" << std::setw(13) << "Efull"
              << std::setw(13) << "Nb" << std::setw(13) << "Sfull" << std::setw(13) << "EtotSurf"
              << std::setw(13) << "elements" << std::setw(10) << "susp." << std::setw(13)
              << "%cut" << std::endl;
    std::cout << std::setw(10) << h->getTau() << std::setw(13) << t.E << std::setw(13) << t.Efull
              << std::setw(13) << ci.nbSurf << std::setw(13) << t.S << std::setw(13)
              << ci.EtotSurf << std::endl;
    std::cout << "corona elements : " << ci.nelements << std::endl;
    if (P.vorticityOn) h->writeBeta(beta.c_str(), true);  // src/main.cpp:391
  }
  do {
    const int nSubSteps = h->advance(P.dtau, P.etamin, P.etamax, P.nz);
    if (nSubSteps > 1) std::cout << "timestep reduced by " << nSubSteps << std::endl;
    const vhb::Totals t = h->totals();
    const vh_surface_info si = h->surface();
    h->writeSurface(fo_unf.c_str(), P.freezeoutExtend);
    if (P.vorticityOn) h->writeBeta(beta.c_str(), false);
    nelements = si.nelements;
    // the line Fluid::outputSurface prints (src/fld.cpp:854-857)
    std::cout << std::setw(10) << h->getTau() << std::setw(13) << t.E << std::setw(13) << t.Efull
              << std::setw(13) << si.nbSurf << std::setw(13) << t.S << std::setw(13)
              << si.EtotSurf << std::setw(10) << si.nelements << std::setw(10) << si.nsusp
              << std::setw(13) << (float)t.nCoreCutCells / (float)t.nCoreCells << std::endl;
    nloops++;
    if (h->getTau() >= P.tauResize && !resized) {
      std::cout << "grid resize\n";
      f = vhb::expandGrid2x(h, eos, eosH, trcoeff);
      resized = true;
    }
  } while (h->getTau() < P.tauMax + 0.0001 && nelements > 0);
  std::rename(fo_unf.c_str(), fo.c_str());  // Fluid::renameOutput

  h->sync();
  unsigned bits = 0;
  vhb::check(vh_error_bits(h->context(), &bits), h->context());
  const std::string out = cl.outputDir + "/final.vhb";
  f->saveSnapshot(out.c_str(), h->getTau(), h->getDtau());
  std::cout << "loops " << nloops << " error_bits " << bits << " final " << out << std::endl;
  delete h;
  delete f;
  delete trcoeff;
  if (eosH != eos) delete eosH;
  delete eos;
  return bits ? 3 : 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    return run(argc, argv);
  } catch (const vhb::Error& e) {
    std::cerr << "vhlle_run: " << e.what() << std::endl;
    return 1;
  }
}
