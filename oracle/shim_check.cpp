// shim_check.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs one event twice from the same initial state: with the reference's
// own Hydro::performStep on a reference Fluid, and through HydroB200
// (include/vhlle_b200_refshim.hpp) on a second reference Fluid, then
// downloads the device state into that Fluid's Cells and lets the
// reference's own Fluid::outputSurface write the freeze-out elements of
// both.  Exits 0 when every cell field is bit-identical and prints the two
// surfaces' element counts; the caller compares the two freezeout.dat files.
//
//   shim_check <ic file> <eos1f file> <steps> <out dir A> <out dir B>
//
// <ic file>: int32 nx ny nz, float64 xmin xmax ymin ymax etamin etamax tau0
// dt ecrit etaS0, then Q[7][N] and m[N] (component-major, x fastest), as
// tests/test_gpu_shim.py writes it.  Built by `make -C oracle shim` from the
// reference's objects (oracle/_ref) and libvhlle_b200.so.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "eos.h"  // before eo1.h
#include "cll.h"
#include "eo1.h"
#include "fld.h"
#include "hdo.h"
#include "inc.h"
#include "trancoeff.h"
#include "vhlle_b200_refshim.hpp"

namespace output {
extern std::ofstream ffreeze, fbeta;
}

namespace {

struct Ic {
  int nx, ny, nz;
  double b[6], tau0, dt, ecrit, etaS0;
  std::vector<double> Q, m;
};

bool read_ic(const char* path, Ic& ic) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  int n[3];
  double d[10];
  bool ok = std::fread(n, sizeof(int), 3, f) == 3 && std::fread(d, sizeof(double), 10, f) == 10;
  if (ok) {
    ic.nx = n[0];
    ic.ny = n[1];
    ic.nz = n[2];
    std::memcpy(ic.b, d, sizeof ic.b);
    ic.tau0 = d[6];
    ic.dt = d[7];
    ic.ecrit = d[8];
    ic.etaS0 = d[9];
    const size_t N = (size_t)ic.nx * ic.ny * ic.nz;
    ic.Q.resize(7 * N);
    ic.m.resize(N);
    ok = std::fread(ic.Q.data(), sizeof(double), 7 * N, f) == 7 * N &&
         std::fread(ic.m.data(), sizeof(double), N, f) == N;
  }
  std::fclose(f);
  return ok;
}

// The EoS1f file's arrays (src/eo1.cpp:21-45) for the device descriptor.
struct Table {
  int ne = 0, nn = 0;
  std::vector<double> eg, ng, p, T, mub;
};

bool read_table(const char* path, Table& t) {
  std::ifstream fin(path);
  double emax, e0, nmax, n0;
  if (!(fin >> emax >> e0 >> nmax >> n0 >> t.ne >> t.nn)) return false;
  t.eg.resize(t.ne);
  t.ng.resize(t.nn);
  for (double& x : t.eg) fin >> x;
  for (double& x : t.ng) fin >> x;
  const size_t n = (size_t)t.ne * t.nn;
  t.p.resize(n);
  t.T.resize(n);
  t.mub.resize(n);
  for (int ie = 0; ie < t.ne; ie++)
    for (int ib = 0; ib < t.nn; ib++) {
      const size_t k = ie + (size_t)t.ne * ib;
      fin >> t.p[k] >> t.T[k] >> t.mub[k];
      if (t.p[k] < 1e-18) t.p[k] = 0.;  // as the reference's reader does
    }
  return (bool)fin;
}

void set_ic(Fluid* f, const Ic& ic) {
  const long N = (long)ic.nx * ic.ny * ic.nz;
  for (int iz = 0; iz < ic.nz; iz++)
    for (int iy = 0; iy < ic.ny; iy++)
      for (int ix = 0; ix < ic.nx; ix++) {
        const long i = ix + (long)ic.nx * (iy + (long)ic.ny * iz);
        double q[7];
        for (int k = 0; k < 7; k++) q[k] = ic.Q[k * N + i];
        Cell* c = f->getCell(ix, iy, iz);
        c->setQ(q);
        c->saveQprev();
        c->setAllM(ic.m[i]);
      }
}

int surface(Fluid* f, const char* dir, double tau0, double tau) {
  if (output::ffreeze.is_open()) output::ffreeze.close();
  std::streambuf* old = std::cout.rdbuf();
  std::ostringstream quiet;
  std::cout.rdbuf(quiet.rdbuf());
  f->initOutput(dir, tau0, true);
  const int n = f->outputSurface(tau, true);
  output::ffreeze.close();
  std::cout.rdbuf(old);
  return n;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s ic eos1f steps outA outB\n", argv[0]);
    return 2;
  }
  Ic ic;
  Table t;
  if (!read_ic(argv[1], ic) || !read_table(argv[2], t)) {
    std::fprintf(stderr, "cannot read the inputs\n");
    return 2;
  }
  const int steps = std::atoi(argv[3]);
  EoS1f eos(argv[2]);
  TransportCoeff tr(ic.etaS0, 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., &eos, 0, 0);
  Fluid fa(&eos, &eos, &tr, ic.nx, ic.ny, ic.nz, ic.b[0], ic.b[1], ic.b[2], ic.b[3], ic.b[4],
           ic.b[5], ic.dt, ic.ecrit);
  Fluid fb(&eos, &eos, &tr, ic.nx, ic.ny, ic.nz, ic.b[0], ic.b[1], ic.b[2], ic.b[3], ic.b[4],
           ic.b[5], ic.dt, ic.ecrit);
  set_ic(&fa, ic);
  set_ic(&fb, ic);

  Hydro ha(&fa, &eos, &tr, ic.tau0, ic.dt);
  vh_grid g{ic.nx, ic.ny, ic.nz, ic.b[0], ic.b[1], ic.b[2], ic.b[3], ic.b[4], ic.b[5]};
  vh_eos d{};
  d.kind = VH_EOS_TABLE;
  d.ne = t.ne;
  d.nn = t.nn;
  d.egrid = t.eg.data();
  d.ngrid = t.ng.data();
  d.p = t.p.data();
  d.T = t.T.data();
  d.mub = t.mub.data();
  try {
    HydroB200 hb(&fb, g, d, &tr, ic.tau0, ic.dt);
    for (int s = 0; s < steps; s++) {
      ha.performStep();
      hb.performStep();
    }
    hb.download();
    if (ha.getTau() != hb.getTau()) {
      std::printf("tau differs: %.17g %.17g\n", ha.getTau(), hb.getTau());
      return 1;
    }
  } catch (const std::exception& e) {
    std::printf("HydroB200 failed: %s\n", e.what());
    return 1;
  }
  long ndiff = 0;
  for (int iz = 0; iz < ic.nz; iz++)
    for (int iy = 0; iy < ic.ny; iy++)
      for (int ix = 0; ix < ic.nx; ix++) {
        Cell* a = fa.getCell(ix, iy, iz);
        Cell* b = fb.getCell(ix, iy, iz);
        double qa[7], qb[7];
        auto cmp = [&](const double* x, const double* y, int n) {
          for (int k = 0; k < n; k++)
            if (!(x[k] == y[k]) && !(std::isnan(x[k]) && std::isnan(y[k]))) ndiff++;
        };
        a->getQ(qa);
        b->getQ(qb);
        cmp(qa, qb, 7);
        a->getQh(qa);
        b->getQh(qb);
        cmp(qa, qb, 7);
        a->getQprev(qa);
        b->getQprev(qb);
        cmp(qa, qb, 7);
        for (int m = 0; m < 4; m++)
          for (int n = 0; n <= m; n++) {
            const double x[2] = {a->getpi(m, n), a->getpiH(m, n)};
            const double y[2] = {b->getpi(m, n), b->getpiH(m, n)};
            cmp(x, y, 2);
          }
        const double x[6] = {a->getPi(), a->getPiH(), a->getM(1), a->getM(2), a->getM(3),
                             a->getViscCorrCutFlag()};
        const double y[6] = {b->getPi(), b->getPiH(), b->getM(1), b->getM(2), b->getM(3),
                             b->getViscCorrCutFlag()};
        cmp(x, y, 6);
      }
  const double tau = ha.getTau();
  const int na = surface(&fa, argv[4], ic.tau0, tau);
  const int nb = surface(&fb, argv[5], ic.tau0, tau);
  std::printf("steps %d tau %.17g differing values %ld elements %d %d\n", steps, tau, ndiff, na,
              nb);
  return ndiff == 0 && na == nb ? 0 : 1;
}
