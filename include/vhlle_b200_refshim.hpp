// vhlle_b200_refshim.hpp -- the binding a maintainer adds to the reference
// tree to run Hydro::performStep (src/hdo.cpp:1016-1134) on the B200 while
// keeping the reference's own Fluid, Cell, EoS and TransportCoeff objects.
//
// Include it after the reference's headers (fld.h, cll.h, eos.h,
// trancoeff.h, inc.h) and link libvhlle_b200.so.  HydroB200 plays Hydro
// (src/hdo.h:7-63): the constructor creates the device context for the
// Fluid's grid and uploads every cell (its Q, Qh, Qprev, pi, piH, Pi, PiH,
// m, viscCorrCut), performStep / setDtau / getDtau / getTau are the
// reference's, and download() writes the device state back into the Cells
// so that the reference's own host code (Fluid::outputSurface,
// outputGnuplot, the VTK writer) reads it.  upload() sends the Cells again
// after the host changed them.
//
// The EoS is a virtual class the device cannot call: the caller lowers it to
// a vh_eos descriptor (for EoS1f, the arrays its constructor reads from its
// file, src/eo1.cpp:21-45).  The grid bounds are the ones the Fluid was
// constructed with (Fluid keeps them private; the device derives dx, dy,
// dz from them exactly as src/fld.cpp:77-79 does).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "vhlle_b200.h"

class HydroB200 {
 public:
  HydroB200(Fluid* f, const vh_grid& grid, const vh_eos& eos, TransportCoeff* tr, double tau0,
            double dt, int device = 0)
      : f_(f), N_((long long)grid.nx * grid.ny * grid.nz) {
    if (grid.nx != f->getNX() || grid.ny != f->getNY() || grid.nz != f->getNZ())
      throw std::invalid_argument("HydroB200: grid size differs from the Fluid's");
    // TransportCoeff's public constants (src/trancoeff.h:8-11); the
    // reference has no zetaSparam 5, so its two parameters stay zero
    vh_trcoeff c{};
    c.etaS0 = tr->etaS0;
    c.zetaS0 = tr->zetaS0;
    c.ah = tr->ah;
    c.al = tr->al;
    c.aRho = tr->aRho;
    c.T0 = tr->T0;
    c.etaSMin = tr->etaSMin;
    c.etaSEpsilonMin = tr->etaSEpsilonMin;
    c.etaSShiftMuB = tr->etaSShiftMuB;
    c.etaSScaleMuB = tr->etaSScaleMuB;
    c.zetaSPeakEpsilon = tr->zetaSPeakEpsilon;
    c.zetaSScaleBeta = tr->zetaSScaleBeta;
    c.zetaSSigmaMinus = tr->zetaSSigmaMinus;
    c.zetaSSigmaPlus = tr->zetaSSigmaPlus;
    c.etaSparam = tr->etaSparam;
    c.zetaSparam = tr->zetaSparam;
    c.zetaSPeakT = 0.;
    c.zetaSWidthT = 0.;
    check(vh_create(&grid, &eos, &c, tau0, dt, device, &ctx_));
    buf_.resize((size_t)kPerCell * N_);
    upload();
  }
  ~HydroB200() { vh_destroy(ctx_); }
  HydroB200(const HydroB200&) = delete;
  HydroB200& operator=(const HydroB200&) = delete;

  // Hydro::performStep: one step on the device (asynchronous; the device
  // error word is checked by download() or sync())
  void performStep() { check(vh_step(ctx_)); }
  void setDtau(double dt) { check(vh_set_dtau(ctx_, dt)); }
  double getDtau() const {
    double dt = 0.;
    check(vh_get_dtau(ctx_, &dt));
    return dt;
  }
  double getTau() const {
    double t = 0.;
    check(vh_get_tau(ctx_, &t));
    return t;
  }
  void sync() { check(vh_sync(ctx_)); }
  vh_ctx* context() { return ctx_; }

  // Cells -> device
  void upload() {
    vh_state_view v = views();
    for (int iz = 0; iz < f_->getNZ(); iz++)
      for (int iy = 0; iy < f_->getNY(); iy++)
        for (int ix = 0; ix < f_->getNX(); ix++) {
          const long long i = index(ix, iy, iz);
          Cell* c = f_->getCell(ix, iy, iz);
          double q[7];
          c->getQ(q);
          put(v.Q, 7, i, q);
          c->getQh(q);
          put(v.Qh, 7, i, q);
          c->getQprev(q);
          put(v.Qprev, 7, i, q);
          for (int a = 0; a < 4; a++)
            for (int b = 0; b <= a; b++) {
              v.pi[index44(a, b) * N_ + i] = c->getpi(a, b);
              v.piH[index44(a, b) * N_ + i] = c->getpiH(a, b);
            }
          v.Pi[i] = c->getPi();
          v.PiH[i] = c->getPiH();
          for (int d = 0; d < 3; d++) v.m[d * N_ + i] = c->getM(d + 1);
          v.viscCorrCut[i] = c->getViscCorrCutFlag();
        }
    check(vh_upload_state(ctx_, &v));
  }

  // device -> Cells (waits for the steps; reports a numerical failure)
  void download() {
    sync();
    vh_state_view v = views();
    check(vh_download_state(ctx_, &v));
    for (int iz = 0; iz < f_->getNZ(); iz++)
      for (int iy = 0; iy < f_->getNY(); iy++)
        for (int ix = 0; ix < f_->getNX(); ix++) {
          const long long i = index(ix, iy, iz);
          Cell* c = f_->getCell(ix, iy, iz);
          double q[7];
          // Cell has no Qprev setter: store it through Q and saveQprev
          get(v.Qprev, 7, i, q);
          c->setQ(q);
          c->saveQprev();
          get(v.Q, 7, i, q);
          c->setQ(q);
          get(v.Qh, 7, i, q);
          c->setQh(q);
          for (int a = 0; a < 4; a++)
            for (int b = 0; b <= a; b++) {
              c->setpi(a, b, v.pi[index44(a, b) * N_ + i]);
              c->setpiH(a, b, v.piH[index44(a, b) * N_ + i]);
            }
          c->setPi(v.Pi[i]);
          c->setPiH(v.PiH[i]);
          // m: above 0.9 every direction is 1 (Cell::addM), so adding each
          // direction's value to zero restores the three values
          c->setAllM(0.);
          for (int d = 0; d < 3; d++) c->addM(d + 1, v.m[d * N_ + i]);
          c->setViscCorrCutFlag(v.viscCorrCut[i]);
        }
  }

 private:
  static constexpr int kPerCell = 7 + 7 + 7 + 10 + 10 + 1 + 1 + 3 + 1;
  Fluid* f_;
  long long N_;
  vh_ctx* ctx_ = nullptr;
  std::vector<double> buf_;

  long long index(int ix, int iy, int iz) const {
    return ix + (long long)f_->getNX() * (iy + (long long)f_->getNY() * iz);
  }
  void put(double* p, int n, long long i, const double* q) const {
    for (int k = 0; k < n; k++) p[k * N_ + i] = q[k];
  }
  void get(const double* p, int n, long long i, double* q) const {
    for (int k = 0; k < n; k++) q[k] = p[k * N_ + i];
  }
  vh_state_view views() {
    double* b = buf_.data();
    vh_state_view v;
    v.Q = b;
    v.Qh = b + 7 * N_;
    v.Qprev = b + 14 * N_;
    v.pi = b + 21 * N_;
    v.piH = b + 31 * N_;
    v.Pi = b + 41 * N_;
    v.PiH = b + 42 * N_;
    v.m = b + 43 * N_;
    v.viscCorrCut = b + 46 * N_;
    return v;
  }
  void check(vh_status st) const {
    if (st != VH_OK) throw std::runtime_error(std::string("HydroB200: ") + vh_last_error(ctx_));
  }
};
