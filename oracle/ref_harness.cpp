// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A thin extern "C" driver around the reference's own, unmodified classes
// (Fluid, Hydro, Cell, EoS1f, TransportCoeff from src/), compiled together
// with them into oracle/_ref/libvhlle_ref.so by oracle/Makefile.  It is the
// pin for the C restatement in vh_oracle.c and the timed CPU baseline.
//
// Harness-owned pieces (not in the reference):
//  * ConformalEoS: p = e/3, T = (e/cnst)^(1/4) evaluated as sqrt(sqrt(.)),
//    muB = 0, the conformal gas of the Gubser-flow workload.  It plays the
//    role of EoSs in its SIMPLE variant (src/eos.cpp:90-110), which the
//    reference only offers at compile time.
//  * The driver loop: performStep is called directly, as the reference main
//    loop does (src/main.cpp:399-428), without the surface-based loop exit.
//  * The initial state is uploaded as conserved Q arrays through Cell::setQ
//    + saveQprev + setAllM, the pattern every reference IC ends with
//    (e.g. src/icGubser.cpp:50-57).
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "eos.h"  // must precede eo1.h, which only forward-declares EoS
#include "cll.h"
#include "cornelius.h"
#include "eo1.h"
#include "eo3.h"
#include "eoChiral.h"
#include "eoHadron.h"
#include "eoSmash.h"
#include "eoAZH.h"
#include "eoCMFe.h"
#include "fld.h"
#include "hdo.h"
#include "ic.h"
#include "icGlissando.h"
#include "icGubser.h"
#include "icPartUrqmd.h"
#include "icTrento.h"
#include "inc.h"
#include "s95p.h"
#include "rmn.h"
#include "trancoeff.h"

// the freeze-out stream Fluid::outputSurface writes to (src/fld.cpp:43-46)
namespace output {
extern std::ofstream ffreeze, fbeta;
}

// the params key glauberVar (oracle/ref_globals.cpp)
extern int glauberVariable;

namespace {

class ConformalEoS : public EoS {
 public:
  explicit ConformalEoS(double cnst) : cnst_(cnst) {}
  void eos(double e, double nb, double nq, double ns, double &T, double &mub,
           double &muq, double &mus, double &p) override {
    (void)nb;
    (void)nq;
    (void)ns;
    p = e / 3.;
    T = e > 0. ? std::sqrt(std::sqrt(e / cnst_)) : 0.;
    mub = muq = mus = 0.;
  }
  double p(double e, double nb, double ns, double nq) override {
    (void)nb;
    (void)ns;
    (void)nq;
    return e / 3.;
  }

 private:
  double cnst_;
};

struct RefRun {
  EoS *eos = nullptr;
  EoS *eosH = nullptr;  // the freeze-out EoS (Fluid's eosH); nullptr: eos
  double bounds[6] = {0, 0, 0, 0, 0, 0};
  double dt = 0;
  TransportCoeff *tr = nullptr;
  Fluid *f = nullptr;
  Hydro *h = nullptr;
  int nx = 0, ny = 0, nz = 0;
  double dx = 0, dy = 0;
  double tau0 = 0, ecrit = 0;
  bool output_open = false;
  bool vorticity = false;
};

}  // namespace

extern "C" {

int ref_abi_version(void) { return 1; }

// tr[14] = etaS0, zetaS0, ah, al, aRho, T0, etaSMin, etaSEpsilonMin,
//          etaSShiftMuB, etaSScaleMuB, zetaSPeakEpsilon, zetaSScaleBeta,
//          zetaSSigmaMinus, zetaSSigmaPlus
void *ref_create(int nx, int ny, int nz, const double *bounds /*6*/,
                 double tau0, double dt, double ecrit, int eos_kind,
                 double conf_cnst, const char *eos_file, const double *tr,
                 int etaSparam, int zetaSparam) {
  RefRun *r = new RefRun;
  if (eos_kind == 0) {
    r->eos = new ConformalEoS(conf_cnst);
  } else if (eos_kind == 2) {
    // EoSChiral reads eos/chiraleos.dat and eos/chiralsmall.dat relative to
    // the working directory (src/eoChiral.cpp:153-156): eos_file names the
    // directory that holds eos/
    char cwd[4096];
    if (!getcwd(cwd, sizeof cwd) || chdir(eos_file) != 0) {
      delete r;
      return nullptr;
    }
    std::streambuf *old = std::cout.rdbuf();
    std::ostringstream quiet;
    std::cout.rdbuf(quiet.rdbuf());
    r->eos = new EoSChiral();
    std::cout.rdbuf(old);
    if (chdir(cwd) != 0) {
      delete r->eos;
      delete r;
      return nullptr;
    }
  } else if (eos_kind == 6 || eos_kind == 7) {
    // EoSAZH reads eos/azhydro0p2/aa{1,2}_{p,t,mb}.dat, EoSCMFe
    // eos/cmfe.dat and eos/cmfe_small.dat, relative to the working directory
    // (src/eoAZH.cpp:110-117, src/eoCMFe.cpp:194-197), as EoSChiral does
    char cwd[4096];
    if (!getcwd(cwd, sizeof cwd) || chdir(eos_file) != 0) {
      delete r;
      return nullptr;
    }
    std::streambuf *old = std::cout.rdbuf();
    std::ostringstream quiet;
    std::cout.rdbuf(quiet.rdbuf());
    if (eos_kind == 6)
      r->eos = new EoSAZH();
    else
      r->eos = new EoSCMFe();
    std::cout.rdbuf(old);
    if (chdir(cwd) != 0) {
      delete r->eos;
      delete r;
      return nullptr;
    }
  } else if (eos_kind == 3) {
    // EoS3f: the header's B is 0 in the files used here, so the
    // constructor's own arguments are not compared with it
    r->eos = new EoS3f(const_cast<char *>(eos_file), 0., 0., 0., 0., 0.);
  } else {
    r->eos = new EoS1f(const_cast<char *>(eos_file));
  }
  r->tr = new TransportCoeff(tr[0], tr[1], tr[2], tr[3], tr[4], tr[5], tr[6],
                             tr[7], tr[8], tr[9], tr[10], tr[11], tr[12],
                             tr[13], r->eos, etaSparam, zetaSparam);
  r->f = new Fluid(r->eos, r->eos, r->tr, nx, ny, nz, bounds[0], bounds[1],
                   bounds[2], bounds[3], bounds[4], bounds[5], dt, ecrit);
  r->h = new Hydro(r->f, r->eos, r->tr, tau0, dt);
  for (int k = 0; k < 6; k++) r->bounds[k] = bounds[k];
  r->dt = dt;
  r->nx = nx;
  r->ny = ny;
  r->nz = nz;
  r->dx = r->f->getDx();
  r->dy = r->f->getDy();
  r->tau0 = tau0;
  r->ecrit = ecrit;
  return r;
}

// EoS::eos of the surface EoS at general charges, as ref_eos_full
void ref_surface_eos_full(void *p, const double *in, int n, double *out) {
  RefRun *r = static_cast<RefRun *>(p);
  EoS *e = r->eosH ? r->eosH : r->eos;
  for (int i = 0; i < n; i++) {
    const double *a = in + 4 * i;
    double *o = out + 5 * i;
    e->eos(a[0], a[1], a[2], a[3], o[1], o[2], o[3], o[4], o[0]);
  }
}

// Fluid's eosH, the EoS of outputSurface and outputCorona (src/fld.cpp:
// 540-542, 870-872: SWAP_EOS), from a table file: kind 4 EoSHadron
// (src/eoHadron.cpp).  The Fluid and Hydro are made again with it, so call
// this before the state is set; kind 5 EoSSmash (src/eoSmash.cpp) takes its
// table's ne, nnb, nnq as the driver passes them (src/main.cpp:308).
// Returns 0, or -1 for an unknown kind.
int ref_set_surface_eos(void *p, int kind, const char *file, int ne, int nnb, int nnq) {
  RefRun *r = static_cast<RefRun *>(p);
  std::streambuf *old = std::cout.rdbuf();
  std::ostringstream quiet;
  std::cout.rdbuf(quiet.rdbuf());
  EoS *eh = nullptr;
  if (kind == 4) eh = new EoSHadron(const_cast<char *>(file));
  if (kind == 5) eh = new EoSSmash(const_cast<char *>(file), ne, nnb, nnq);
  std::cout.rdbuf(old);
  if (!eh) return -1;
  r->eosH = eh;
  const double tau0 = r->h->getTau();
  delete r->h;
  delete r->f;
  r->f = new Fluid(r->eos, r->eosH, r->tr, r->nx, r->ny, r->nz, r->bounds[0], r->bounds[1],
                   r->bounds[2], r->bounds[3], r->bounds[4], r->bounds[5], r->dt, r->ecrit);
  r->h = new Hydro(r->f, r->eos, r->tr, tau0, r->dt);
  return 0;
}

void ref_destroy(void *p) {
  RefRun *r = static_cast<RefRun *>(p);
  if (r->output_open && output::ffreeze.is_open()) output::ffreeze.close();
  if (r->output_open && output::fbeta.is_open()) output::fbeta.close();
  delete r->h;
  delete r->f;
  delete r->tr;
  delete r->eos;
  delete r->eosH;
  delete r;
}

// Q[7][N], pi[10][N], piH[10][N], Pi[N], PiH[N], m[N] (uniform per cell);
// any of pi/piH/Pi/PiH may be null (then zero).
void ref_set_state(void *p, const double *Q, const double *pi,
                   const double *piH, const double *Pi, const double *PiH,
                   const double *m) {
  RefRun *r = static_cast<RefRun *>(p);
  const long N = (long)r->nx * r->ny * r->nz;
  for (int iz = 0; iz < r->nz; iz++)
    for (int iy = 0; iy < r->ny; iy++)
      for (int ix = 0; ix < r->nx; ix++) {
        const long i = ix + (long)r->nx * (iy + (long)r->ny * iz);
        Cell *c = r->f->getCell(ix, iy, iz);
        double q[7];
        for (int k = 0; k < 7; k++) q[k] = Q[k * N + i];
        c->setQ(q);
        c->saveQprev();
        c->setAllM(m[i]);
        for (int a = 0; a < 4; a++)
          for (int b = 0; b <= a; b++) {
            const int k = index44(a, b);
            c->setpi(a, b, pi ? pi[k * N + i] : 0.);
            c->setpiH(a, b, piH ? piH[k * N + i] : 0.);
          }
        c->setPi(Pi ? Pi[i] : 0.);
        c->setPiH(PiH ? PiH[i] : 0.);
      }
}

void ref_step(void *p, int nsteps) {
  RefRun *r = static_cast<RefRun *>(p);
  for (int s = 0; s < nsteps; s++) r->h->performStep();
}

double ref_tau(void *p) { return static_cast<RefRun *>(p)->h->getTau(); }

// expandGrid2x (src/main.cpp:246-271) restated over the reference's own
// Fluid/Cell/Hydro objects (main.cpp is not compiled into the harness since
// it holds main()).  Returns 1 when resized, 0 when the grid is not
// symmetric, -1 when the doubled step would fail Hydro::setDtau's check.
int ref_resize2x(void *p) {
  RefRun *r = static_cast<RefRun *>(p);
  Fluid *f = r->f;
  if (f->getX(0) + f->getX(f->getNX() - 1) > 0.001 ||
      f->getY(0) + f->getY(f->getNY() - 1) > 0.001)
    return 0;
  Fluid *fnew = new Fluid(r->eos, r->eosH ? r->eosH : r->eos, r->tr, f->getNX(), f->getNY(), f->getNZ(),
                          2.0 * f->getX(0), 2.0 * f->getX(f->getNX() - 1),
                          2.0 * f->getY(0), 2.0 * f->getY(f->getNY() - 1), f->getZ(0),
                          f->getZ(f->getNZ() - 1), 2.0 * r->h->getDtau(), f->geteCrit());
  const double dt2 = 2.0 * r->h->getDtau();
  if (dt2 > fnew->getDx() / 2. || dt2 > fnew->getDy() / 2.) {
    delete fnew;
    return -1;
  }
  for (int ix = 0; ix < f->getNX(); ix++)
    for (int iy = 0; iy < f->getNY(); iy++)
      for (int iz = 0; iz < f->getNZ(); iz++)
        fnew->getCell(ix, iy, iz)->importVars(f->getCell(2 * (ix - f->getNX() / 2) + f->getNX() / 2,
                                                         2 * (iy - f->getNY() / 2) + f->getNY() / 2, iz));
  // src/main.cpp:257,264-265: the new fluid's cells get zero dbeta
  if (r->vorticity) fnew->enableVorticity();
  r->h->setFluid(fnew);
  r->h->setDtau(dt2);
  delete f;
  r->f = fnew;
  r->dx = fnew->getDx();
  r->dy = fnew->getDy();
  return 1;
}

// The substep block of the driver loop (src/main.cpp:405-419) with
// performStep; returns the substep count.
int ref_advance(void *p, double dtau, double etamin, double etamax, int nz) {
  RefRun *r = static_cast<RefRun *>(p);
  Hydro *h = r->h;
  int nSubSteps = 1;
  while (dtau / nSubSteps > 1.0 * h->getTau() * (etamax - etamin) / (nz - 1)) nSubSteps *= 2;
  if (nSubSteps > 1) {
    h->setDtau(h->getDtau() / nSubSteps);
    for (int j = 0; j < nSubSteps; j++) h->performStep();
    h->setDtau(h->getDtau() * nSubSteps);
  } else {
    h->performStep();
  }
  return nSubSteps;
}

double ref_dtau(void *p) { return static_cast<RefRun *>(p)->h->getDtau(); }

// out[9] = getX(0), getX(nx-1), getY(0), getY(ny-1), getZ(0), getZ(nz-1),
//          dx, dy, dz of the current fluid
void ref_grid(void *p, double *out) {
  Fluid *f = static_cast<RefRun *>(p)->f;
  out[0] = f->getX(0);
  out[1] = f->getX(f->getNX() - 1);
  out[2] = f->getY(0);
  out[3] = f->getY(f->getNY() - 1);
  out[4] = f->getZ(0);
  out[5] = f->getZ(f->getNZ() - 1);
  out[6] = f->getDx();
  out[7] = f->getDy();
  out[8] = f->getDz();
}

// Hydro::setDtau exits when dt > dx/2; refuse that here instead.
int ref_set_dtau(void *p, double dt) {
  RefRun *r = static_cast<RefRun *>(p);
  if (dt > r->dx / 2. || dt > r->dy / 2.) return 1;
  r->h->setDtau(dt);
  return 0;
}

// out arrays: component-major, any may be null.
void ref_get_state(void *p, double *Q, double *Qh, double *Qprev, double *pi,
                   double *piH, double *Pi, double *PiH, double *m,
                   double *vcc) {
  RefRun *r = static_cast<RefRun *>(p);
  const long N = (long)r->nx * r->ny * r->nz;
  for (int iz = 0; iz < r->nz; iz++)
    for (int iy = 0; iy < r->ny; iy++)
      for (int ix = 0; ix < r->nx; ix++) {
        const long i = ix + (long)r->nx * (iy + (long)r->ny * iz);
        Cell *c = r->f->getCell(ix, iy, iz);
        double q[7];
        if (Q) {
          c->getQ(q);
          for (int k = 0; k < 7; k++) Q[k * N + i] = q[k];
        }
        if (Qh) {
          c->getQh(q);
          for (int k = 0; k < 7; k++) Qh[k * N + i] = q[k];
        }
        if (Qprev) {
          c->getQprev(q);
          for (int k = 0; k < 7; k++) Qprev[k * N + i] = q[k];
        }
        for (int a = 0; a < 4; a++)
          for (int b = 0; b <= a; b++) {
            const int k = index44(a, b);
            if (pi) pi[k * N + i] = c->getpi(a, b);
            if (piH) piH[k * N + i] = c->getpiH(a, b);
          }
        if (Pi) Pi[i] = c->getPi();
        if (PiH) PiH[i] = c->getPiH();
        if (m)
          for (int d = 0; d < 3; d++) m[d * N + i] = c->getM(d + 1);
        if (vcc) vcc[i] = c->getViscCorrCutFlag();
      }
}

// transformPV on n row-major states Q[n][7] -> out[n][8]
void ref_transform_pv(void *p, const double *Q, int n, double *out) {
  RefRun *r = static_cast<RefRun *>(p);
  for (int i = 0; i < n; i++) {
    double q[7];
    for (int k = 0; k < 7; k++) q[k] = Q[7 * i + k];
    double *o = out + 8 * i;
    transformPV(r->eos, q, o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7]);
  }
}

// Cell::setPrimVar (src/cll.cpp:222-241) with the run's EoS, through a
// scratch Cell: in[n][8] = tau, e, nb, nq, ns, vx, vy, vz -> out[n][7] = the
// Q it stores.  The IC modules end with this call for every cell.
void ref_set_prim_var(void *p, const double *in, int n, double *out) {
  RefRun *r = static_cast<RefRun *>(p);
  Cell c;
  for (int i = 0; i < n; i++) {
    const double *a = in + 8 * i;
    c.setPrimVar(r->eos, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7]);
    c.getQ(out + 7 * i);
  }
}

// TransportCoeff::getEta + getTau: in[n][6] = e, nb, T, muB, s, p ->
// out[n][4] = eta/s, zeta/s, tau_pi, tau_Pi
void ref_transport_eval(void *p, const double *in, int n, double *out) {
  RefRun *r = static_cast<RefRun *>(p);
  for (int i = 0; i < n; i++) {
    const double *a = in + 6 * i;
    double *o = out + 4 * i;
    r->tr->getEta(a[0], a[1], a[2], a[3], a[4], a[5], o[0], o[1]);
    r->tr->getTau(a[0], a[1], a[2], a[3], a[4], a[5], o[2], o[3]);
  }
}

// EoS::eos -> out[n][3] = p, T, mub ; s_out[n] = EoS::s
void ref_eos(void *p, const double *e, const double *nb, int n, double *out,
             double *s_out) {
  RefRun *r = static_cast<RefRun *>(p);
  for (int i = 0; i < n; i++) {
    double T, mub, muq, mus, pp;
    r->eos->eos(e[i], nb[i], 0., 0., T, mub, muq, mus, pp);
    out[3 * i] = pp;
    out[3 * i + 1] = T;
    out[3 * i + 2] = mub;
    if (s_out) s_out[i] = r->eos->s(e[i], nb[i], 0., 0.);
  }
}

// EoS::eos at general charges: in[n][4] = e, nb, nq, ns -> out[n][5] = p,
// T, muB, muQ, muS
void ref_eos_full(void *p, const double *in, int n, double *out) {
  RefRun *r = static_cast<RefRun *>(p);
  for (int i = 0; i < n; i++) {
    const double *a = in + 4 * i;
    double *o = out + 5 * i;
    r->eos->eos(a[0], a[1], a[2], a[3], o[1], o[2], o[3], o[4], o[0]);
  }
}

// EoS::eos with muS, EoS::p and EoS::s (nq = ns = 0) on arrays:
// out[n][6] = p, T, muB, muS, p(), s
void ref_eos6(void *p, const double *e, const double *nb, int n, double *out) {
  RefRun *r = static_cast<RefRun *>(p);
  for (int i = 0; i < n; i++) {
    double T, mub, muq, mus, pp;
    r->eos->eos(e[i], nb[i], 0., 0., T, mub, muq, mus, pp);
    double *o = out + 6 * i;
    o[0] = pp;
    o[1] = T;
    o[2] = mub;
    o[3] = mus;
    o[4] = r->eos->p(e[i], nb[i], 0., 0.);
    o[5] = r->eos->s(e[i], nb[i], 0., 0.);
  }
}

// The interior totals of Fluid::outputSurface (src/fld.cpp:544-604, scaled
// at :846-851), accumulated here with the reference's own Fluid/Cell/EoS
// methods in its loop order, at full precision (outputSurface itself prints
// them with 6 digits).  out[16]: E, Efull, Nb1, Nb2, S, Px, vt_num, vt_den,
// vxvy_num, vxvy_den, pi0x_num, pi0x_den, txxyy_num, txxyy_den,
// nCoreCells, nCoreCutCells.
void ref_totals(void *p, double tau, double *out) {
  RefRun *r = static_cast<RefRun *>(p);
  Fluid *f = r->f;
  const int nx = r->nx, ny = r->ny, nz = r->nz;
  const double dx = f->getDx(), dy = f->getDy(), dz = f->getDz();
  const bool visc = r->tr->isViscous();
  double E = 0., Efull = 0., S = 0., Px = 0., vt_num = 0., vt_den = 0.,
         vxvy_num = 0., vxvy_den = 0., pi0x_num = 0., pi0x_den = 0.,
         txxyy_num = 0., txxyy_den = 0., Nb1 = 0., Nb2 = 0.;
  int nCoreCells = 0, nCoreCutCells = 0;
  for (int ix = 2; ix < nx - 2; ix++)
    for (int iy = 2; iy < ny - 2; iy++)
      for (int iz = 2; iz < nz - 2; iz++) {
        Cell *c = f->getCell(ix, iy, iz);
        double e, nb, nq, ns, vx, vy, vz, t, mub, muq, mus, p, Q[7];
        // outputSurface computes these after swapping in Fluid's eosH
        // (src/fld.cpp:540-550): Fluid::getCMFvariables (src/fld.cpp:50-60)
        // with that EoS
        EoS *eh = r->eosH ? r->eosH : r->eos;
        {
          double pp, vzz;
          c->getPrimVar(eh, tau, e, pp, nb, nq, ns, vx, vy, vzz);
          const double etac = f->getZ(c->getZ());
          vz = etac + 1. / 2. * log((1. + vzz) / (1. - vzz));
          vx = vx * cosh(vz - etac) / cosh(vz);
          vy = vy * cosh(vz - etac) / cosh(vz);
        }
        c->getQ(Q);
        eh->eos(e, nb, nq, ns, t, mub, muq, mus, p);
        double s = eh->s(e, nb, nq, ns);
        const double eta = f->getZ(iz);
        const double cosh_int = (sinh(eta + 0.5 * dz) - sinh(eta - 0.5 * dz)) / dz;
        const double sinh_int = (cosh(eta + 0.5 * dz) - cosh(eta - 0.5 * dz)) / dz;
        E += tau * (e + p) / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz)) *
                 (cosh_int - tanh(vz) * sinh_int) -
             tau * p * cosh_int;
        Nb1 += Q[NB_];
        Nb2 += tau * nb * (cosh_int - tanh(vz) * sinh_int) /
               sqrt(1. - vx * vx - vy * vy - tanh(vz) * tanh(vz));
        Efull += tau * (e + p) / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz)) *
                     (cosh(eta) - tanh(vz) * sinh(eta)) -
                 tau * p * cosh(eta);
        if (visc) Efull += tau * c->getpi(0, 0) * cosh(eta) + tau * c->getpi(0, 3) * sinh(eta);
        if (e > r->ecrit) {
          nCoreCells++;
          if (c->getViscCorrCutFlag() < 0.9) nCoreCutCells++;
        }
        const double gmumu[4] = {1., -1., -1., -1.};
        double deltas = 0.;
        if (visc)
          for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++)
              deltas += pow(c->getpi(i, j), 2) * gmumu[i] * gmumu[j];
        if (t > 0.02) {
          s += 1.5 * deltas / ((e + p) * t);
          S += tau * s * (cosh_int - tanh(vz) * sinh_int) /
               sqrt(1. - vx * vx - vy * vy - tanh(vz) * tanh(vz));
        }
        Px += tau * (e + p) * vx / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz));
        if (iz > nz / 2 - 3 and iz < nz / 2 + 3) {
          vxvy_num += e * (fabs(vx) - fabs(vy));
          vxvy_den += e;
          vt_den += e / sqrt(1. - vx * vx - vy * vy);
          vt_num += e / sqrt(1. - vx * vx - vy * vy) * sqrt(vx * vx + vy * vy);
          txxyy_num += (e + p) / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz)) *
                       (vx * vx - vy * vy);
          txxyy_den += (e + p) / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz)) *
                           (vx * vx + vy * vy) +
                       2. * p;
        }
        pi0x_num += e / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz)) * fabs(c->getpi(0, 1));
        pi0x_den += e / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz));
      }
  E = E * dx * dy * dz;
  Efull = Efull * dx * dy * dz;
  S = S * dx * dy * dz;
  Nb1 *= dx * dy * dz;
  Nb2 *= dx * dy * dz;
  const double v[16] = {E, Efull, Nb1, Nb2, S, Px, vt_num, vt_den, vxvy_num, vxvy_den,
                        pi0x_num, pi0x_den, txxyy_num, txxyy_den, (double)nCoreCells,
                        (double)nCoreCutCells};
  for (int k = 0; k < 16; k++) out[k] = v[k];
}

// Fluid::outputSurface itself (src/fld.cpp:517-874).  The first call opens
// `dir`/freezeout.dat.unfinished (Fluid::initOutput with hsOnly = true).
// Returns the number of surface elements; the line outputSurface prints
// (tau E Efull nbSurf S EtotSurf nelements nsusp cut-fraction, 6 digits) is
// copied into `line`.
int ref_output_surface(void *p, const char *dir, int extendFO, char *line, int linelen) {
  RefRun *r = static_cast<RefRun *>(p);
  std::streambuf *old = std::cout.rdbuf();
  std::ostringstream cap;
  std::cout.rdbuf(cap.rdbuf());
  if (!r->output_open) {
    // the freeze-out stream is a process-wide global: one run at a time
    if (output::ffreeze.is_open()) output::ffreeze.close();
    if (output::fbeta.is_open()) output::fbeta.close();
    r->f->initOutput(dir, r->tau0, true);
    r->output_open = true;
  }
  const int n = r->f->outputSurface(r->h->getTau(), extendFO != 0);
  output::ffreeze.flush();
  if (output::fbeta.is_open()) output::fbeta.flush();
  std::cout.rdbuf(old);
  const std::string all = cap.str();
  // the totals line is the last non-empty line
  std::string last;
  std::istringstream in(all);
  for (std::string l; std::getline(in, l);)
    if (!l.empty()) last = l;
  if (line && linelen > 0) {
    strncpy(line, last.c_str(), linelen - 1);
    line[linelen - 1] = 0;
  }
  return n;
}

// Fluid::outputCorona at the current tau into the same freeze-out stream;
// returns the number of corona elements (the "corona elements : n" line)
// and copies the totals line it prints (the second-to-last line).
int ref_output_corona(void *p, const char *dir, int extendFO, char *line, int linelen) {
  RefRun *r = static_cast<RefRun *>(p);
  std::streambuf *old = std::cout.rdbuf();
  std::ostringstream cap;
  std::cout.rdbuf(cap.rdbuf());
  if (!r->output_open) {
    if (output::ffreeze.is_open()) output::ffreeze.close();
    r->f->initOutput(dir, r->tau0, true);
    r->output_open = true;
  }
  r->f->outputCorona(r->h->getTau(), extendFO != 0);
  output::ffreeze.flush();
  std::cout.rdbuf(old);
  std::vector<std::string> lines;
  std::istringstream in(cap.str());
  for (std::string l; std::getline(in, l);)
    if (!l.empty()) lines.push_back(l);
  int n = -1;
  if (!lines.empty()) {
    const std::string &last = lines.back();
    const size_t k = last.find(':');
    if (k != std::string::npos) n = atoi(last.c_str() + k + 1);
  }
  if (line && linelen > 0) {
    const std::string t = lines.size() >= 2 ? lines[lines.size() - 2] : std::string();
    strncpy(line, t.c_str(), linelen - 1);
    line[linelen - 1] = 0;
  }
  return n;
}

// Hydro::enableVorticity (src/hdo.cpp:60-64): dbeta in every cell, written
// by ISformal from the next step on, and beta.dat lines from outputSurface
// (the file opens with the freeze-out output, so call this before the first
// ref_output_surface).
void ref_enable_vorticity(void *p) {
  RefRun *r = static_cast<RefRun *>(p);
  r->h->enableVorticity();
  r->vorticity = true;
}

// Cell::getDbeta of every cell: out[(4 mu + nu) * N + i], i x-fastest.
void ref_get_dbeta(void *p, double *out) {
  RefRun *r = static_cast<RefRun *>(p);
  const long N = (long)r->nx * r->ny * r->nz;
  for (int iz = 0; iz < r->nz; iz++)
    for (int iy = 0; iy < r->ny; iy++)
      for (int ix = 0; ix < r->nx; ix++) {
        const long i = ix + (long)r->nx * (iy + (long)r->ny * iz);
        Cell *c = r->f->getCell(ix, iy, iz);
        for (int a = 0; a < 4; a++)
          for (int b = 0; b < 4; b++) out[(4 * a + b) * N + i] = c->getDbeta(a, b);
      }
}

// Fluid::printDbetaHeader (src/fld.cpp:174-188) into beta.dat: 0, or -1
// when the reference throws (no corona count yet).
int ref_print_dbeta_header(void *p) {
  RefRun *r = static_cast<RefRun *>(p);
  try {
    r->f->printDbetaHeader();
  } catch (const std::exception &) {
    return -1;
  }
  if (output::fbeta.is_open()) output::fbeta.flush();
  return 0;
}

// The reference's Cornelius class on one hypercube: cube[it*8+jx*4+jy*2+jz],
// dx[4]; writes up to 10 centroids and normals, returns the element count.
int ref_cornelius4d(const double *cube, const double *dx, double E0, double *cent,
                    double *norm) {
  static Cornelius *cor = nullptr;
  if (!cor) cor = new Cornelius;
  double arrayDx[4] = {dx[0], dx[1], dx[2], dx[3]};
  cor->init(4, E0, arrayDx);
  double ****c = new double ***[2];
  for (int i = 0; i < 2; i++) {
    c[i] = new double **[2];
    for (int j = 0; j < 2; j++) {
      c[i][j] = new double *[2];
      for (int k = 0; k < 2; k++) {
        c[i][j][k] = new double[2];
        for (int l = 0; l < 2; l++) c[i][j][k][l] = cube[i * 8 + j * 4 + k * 2 + l];
      }
    }
  }
  cor->find_surface_4d(c);
  const int n = cor->get_Nelements();
  for (int e = 0; e < n; e++)
    for (int d = 0; d < 4; d++) {
      cent[e * 4 + d] = cor->get_centroid_elem(e, d);
      norm[e * 4 + d] = cor->get_normal_elem(e, d);
    }
  for (int i = 0; i < 2; i++) {
    for (int j = 0; j < 2; j++) {
      for (int k = 0; k < 2; k++) delete[] c[i][j][k];
      delete[] c[i][j];
    }
    delete[] c[i];
  }
  delete[] c;
  return n;
}

// One of the reference's IC modules run on a fresh Fluid of the run's grid,
// as the driver does (src/main.cpp:320-366): model 2 IC (the entropy or energy
// table of file, scaled by s0scale; glauber_var sets glauberVar), 3
// IcPartUrqmd (file, the widths Rgt and Rgz), 4 ICGubser, 5 IcGlissando, 7
// IcTrento (file and the setup name).  Returns
// every cell's Q and Qprev [7][N] and m [N] (its three directions are
// equal), in the grid order (ix fastest), or -1 for another model.  The
// modules' console output is discarded.
int ref_ic(void *p, int model, const char *file, const char *setup, double s0scale,
           int glauber_var, double Rgt, double Rgz, double *Q, double *Qprev, double *m) {
  RefRun *r = static_cast<RefRun *>(p);
  if (model != 2 && model != 3 && model != 4 && model != 5 && model != 7) return -1;
  // a fresh Fluid (and its Hydro), as the driver builds before the IC
  delete r->h;
  delete r->f;
  r->f = new Fluid(r->eos, r->eosH ? r->eosH : r->eos, r->tr, r->nx, r->ny, r->nz, r->bounds[0],
                   r->bounds[1], r->bounds[2], r->bounds[3], r->bounds[4], r->bounds[5], r->dt,
                   r->ecrit);
  r->h = new Hydro(r->f, r->eos, r->tr, r->tau0, r->dt);
  std::streambuf *old = std::cout.rdbuf();
  std::ostringstream quiet;
  std::cout.rdbuf(quiet.rdbuf());
  if (model == 2) {
    glauberVariable = glauber_var;
    IC ic(file, s0scale);
    ic.setIC(r->f, r->eos, r->tau0);
  } else if (model == 3) {
    IcPartUrqmd ic(r->f, file, Rgt, Rgz, r->tau0);
    ic.setIC(r->f, r->eos);
  } else if (model == 4) {
    ICGubser ic;
    ic.setIC(r->f, r->eos, r->tau0);
  } else if (model == 5) {
    IcGlissando ic(r->f, file, r->tau0, setup);
    ic.setIC(r->f, r->eos);
  } else {
    IcTrento ic(r->f, file, r->tau0, setup);
    ic.setIC(r->f, r->eos);
  }
  std::cout.rdbuf(old);
  const long N = (long)r->nx * r->ny * r->nz;
  for (int iz = 0; iz < r->nz; iz++)
    for (int iy = 0; iy < r->ny; iy++)
      for (int ix = 0; ix < r->nx; ix++) {
        const long i = ix + (long)r->nx * (iy + (long)r->ny * iz);
        Cell *c = r->f->getCell(ix, iy, iz);
        double q[7], qp[7];
        c->getQ(q);
        c->getQprev(qp);
        for (int k = 0; k < 7; k++) {
          Q[k * N + i] = q[k];
          Qprev[k * N + i] = qp[k];
        }
        m[i] = c->getM(X_);
      }
  return 0;
}

// s95p::s95p_e (src/s95p.cpp:34-41) of n entropy densities
void ref_s95p_e(const double *s, int n, double *out) {
  for (int i = 0; i < n; i++) out[i] = s95p::s95p_e(s[i]);
}

// Fluid::updateM alone (test of the vacuum-front rule)
void ref_update_m(void *p, double tau, double dt) {
  static_cast<RefRun *>(p)->f->updateM(tau, dt);
}

}  // extern "C"
