// vhlle_b200.hpp -- C++ host layer over the C ABI (vhlle_b200.h), keeping
// the reference's class surface so that a vHLLE-style driver changes only
// its includes: EoS1f (src/eo1.h), TransportCoeff (src/trancoeff.h), Fluid
// (src/fld.h) with Cell-level accessors (src/cll.h), Hydro (src/hdo.h) and
// the params-file reader (src/main.cpp:70-156).
//
// Differences a caller sees:
//  * Hydro owns a device copy of the Fluid's cells.  performStep() runs on
//    the GPU; the Fluid's host arrays are refreshed by Hydro::sync() (and
//    uploaded again by setFluid or after the caller edits cells and calls
//    upload()).
//  * Conditions the reference stops on with exit() throw vhb::Error.
//  * EoS objects must be lowerable to the device (conformal gas or an EoS1f
//    table); their host p()/eos() follow the reference for initial states.
#pragma once

#include <algorithm>
#include <limits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "vhlle_b200.h"

namespace vhb {

enum { T_ = 0, X_ = 1, Y_ = 2, Z_ = 3, NB_ = 4, NQ_ = 5, NS_ = 6 };

struct Error : std::runtime_error {
  int status;
  Error(int st, const std::string& m) : std::runtime_error(m), status(st) {}
};

inline void check(vh_status st, vh_ctx* ctx) {
  if (st != VH_OK) throw Error(st, vh_last_error(ctx));
}

// index44, src/cll.cpp:22-31
inline int index44(int i, int j) { return (j < i) ? (i * (i + 1)) / 2 + j : (j * (j + 1)) / 2 + i; }

// ------------------------------------------------------------------- EoS
// Abstract EoS (src/eos.h:21-38) restricted to what the device can evaluate.
class EoS {
 public:
  virtual ~EoS() {}
  virtual void eos(double e, double nb, double nq, double ns, double& T, double& mub,
                   double& muq, double& mus, double& p) const = 0;
  virtual double p(double e, double nb, double nq, double ns) const {
    double T, mub, muq, mus, pp;
    eos(e, nb, nq, ns, T, mub, muq, mus, pp);
    return pp;
  }
  // EoS::s, src/eos.cpp:18-25
  double s(double e, double nb, double nq, double ns) const {
    double T, mub, muq, mus, p;
    eos(e, nb, nq, ns, T, mub, muq, mus, p);
    return T > 0.0 ? (e + p - mub * nb - muq * nq - mus * ns) / T : 0.;
  }
  virtual vh_eos descriptor() const = 0;
};

// Conformal gas p = e/3, e = cnst T^4.
class EoSConformal : public EoS {
  double cnst_;

 public:
  explicit EoSConformal(double cnst) : cnst_(cnst) {}
  void eos(double e, double, double, double, double& T, double& mub, double& muq, double& mus,
           double& p) const override {
    p = e / 3.;
    T = e > 0. ? std::sqrt(std::sqrt(e / cnst_)) : 0.;
    mub = muq = mus = 0.;
  }
  vh_eos descriptor() const override {
    vh_eos d{};
    d.kind = VH_EOS_CONFORMAL;
    d.conf_cnst = cnst_;
    return d;
  }
};

// EoS1f (src/eo1.cpp:21-123): (e, nb) table read from the same file format.
class EoS1f : public EoS {
  int ne_ = 0, nn_ = 0;
  std::vector<double> eg_, ng_, p_, T_, mub_;

  static void bracket(const std::vector<double>& g, double x, int& k1, double& u) {
    int n = (int)g.size(), lo = 0, hi = n - 1;
    while (hi - lo > 1) {
      const int k = (lo + hi) / 2;
      if (x < g[k])
        hi = k;
      else
        lo = k;
    }
    k1 = lo;
    if (k1 > n - 2) k1 = n - 2;
    if (k1 < 0) k1 = 0;
    u = (x - g[lo]) / (g[hi] - g[lo]);
  }

 public:
  explicit EoS1f(const char* filename) {
    std::ifstream fin(filename);
    if (!fin) throw Error(VH_ERR_ARG, std::string("EoS1f: cannot open ") + filename);
    double emax, e0, nmax, n0;
    fin >> emax >> e0 >> nmax >> n0 >> ne_ >> nn_;
    if (!fin || ne_ < 2 || nn_ < 2) throw Error(VH_ERR_ARG, "EoS1f: bad table header");
    eg_.resize(ne_);
    ng_.resize(nn_);
    for (double& v : eg_) fin >> v;
    for (double& v : ng_) fin >> v;
    p_.resize((size_t)ne_ * nn_);
    T_.resize(p_.size());
    mub_.resize(p_.size());
    for (int ie = 0; ie < ne_; ie++)
      for (int inb = 0; inb < nn_; inb++) {
        const size_t k = ie + (size_t)ne_ * inb;
        fin >> p_[k] >> T_[k] >> mub_[k];
        if (p_[k] < 1e-18) p_[k] = 0.;
      }
    if (!fin) throw Error(VH_ERR_ARG, "EoS1f: truncated table");
  }
  void eos(double e, double nb, double, double, double& T, double& mub, double& muq,
           double& mus, double& p) const override {
    int ie, inb;
    double ue, un;
    bracket(eg_, e, ie, ue);
    bracket(ng_, nb, inb, un);
    const double we[2] = {1. - ue, ue}, wn[2] = {1. - un, un};
    T = mub = muq = mus = p = 0.;
    for (int je = 0; je < 2; je++)
      for (int jn = 0; jn < 2; jn++) {
        const size_t k = (ie + je) + (size_t)ne_ * (inb + jn);
        p += we[je] * wn[jn] * p_[k];
        T += we[je] * wn[jn] * T_[k];
        mub += we[je] * wn[jn] * mub_[k];
      }
    if (p < 0.) p = 0.;
  }
  vh_eos descriptor() const override {
    vh_eos d{};
    d.kind = VH_EOS_TABLE;
    d.ne = ne_;
    d.nn = nn_;
    d.egrid = eg_.data();
    d.ngrid = ng_.data();
    d.p = p_.data();
    d.T = T_.data();
    d.mub = mub_.data();
    return d;
  }
};

// EoS3f (src/eo3.cpp:21-175): the (e, nb, nq, ns) table with one n grid
// for the three charges.  Reads the reference's file (the header constants
// B, volex0, delta0, aaa, bbb are compared with the constructor's when the
// file's B is positive, as the reference does, with an exception in place
// of its exit); eos() interpolates the 16 corners in the reference's order.
class EoS3f : public EoS {
  int ne_ = 0, nn_ = 0;
  std::vector<double> eg_, ng_, p_, T_, mub_, muq_, mus_;

  // getue / getun (src/eo3.cpp:98-130): the e index is clamped from above
  // only, the weight comes from the unclamped bracket
  static void bracket(const std::vector<double>& g, double x, bool clamp_low, int& ix,
                      double& u) {
    int n = (int)g.size(), k1 = 0, k2 = n - 1;
    while (k2 - k1 > 1) {
      const int k = (k1 + k2) / 2;
      if (x < g[k])
        k2 = k;
      else
        k1 = k;
    }
    ix = k1 > n - 2 ? n - 2 : k1;
    if (clamp_low && ix < 0) ix = 0;
    u = (x - g[k1]) / (g[k2] - g[k1]);
  }
  size_t index(int ie, int ib, int iq, int is) const {
    return ie + (size_t)ne_ * ib + (size_t)ne_ * nn_ * iq + (size_t)ne_ * nn_ * nn_ * is;
  }

 public:
  EoS3f(const char* filename, double B, double volex0, double delta0, double aaa, double bbb) {
    std::ifstream fin(filename);
    if (!fin) throw Error(VH_ERR_ARG, std::string("EoS3f: cannot open ") + filename);
    double h[5];
    for (double& v : h) fin >> v;
    const double want[5] = {B, volex0, delta0, aaa, bbb};
    if (h[0] > 0)
      for (int k = 0; k < 5; k++)
        if (std::fabs(h[k] - want[k]) > 1e-5)
          throw Error(VH_ERR_ARG, "EoS3f: the table's header constants differ from the arguments");
    double emax, e0, nmax, n0;
    fin >> emax >> e0 >> nmax >> n0 >> ne_ >> nn_;
    if (!fin || ne_ < 2 || nn_ < 2) throw Error(VH_ERR_ARG, "EoS3f: bad table header");
    eg_.resize(ne_);
    ng_.resize(nn_);
    for (double& v : eg_) fin >> v;
    for (double& v : ng_) fin >> v;
    const size_t n = (size_t)ne_ * nn_ * nn_ * nn_;
    for (auto* t : {&p_, &T_, &mub_, &muq_, &mus_}) t->resize(n);
    for (int ie = 0; ie < ne_; ie++)
      for (int ib = 0; ib < nn_; ib++)
        for (int iq = 0; iq < nn_; iq++)
          for (int is = 0; is < nn_; is++) {
            const size_t k = index(ie, ib, iq, is);
            fin >> p_[k] >> T_[k] >> mub_[k] >> muq_[k] >> mus_[k];
            if (p_[k] < 1e-18) p_[k] = 0.;
          }
    if (!fin) throw Error(VH_ERR_ARG, "EoS3f: truncated table");
  }
  void eos(double e, double nb, double nq, double ns, double& T, double& mub, double& muq,
           double& mus, double& p) const override {
    int ie, ib, iq, is;
    double ue, ub, uq, us;
    bracket(eg_, e, false, ie, ue);
    bracket(ng_, nb, true, ib, ub);
    bracket(ng_, nq, true, iq, uq);
    bracket(ng_, ns, true, is, us);
    const double we[2] = {1. - ue, ue}, wb[2] = {1. - ub, ub};
    const double wq[2] = {1. - uq, uq}, ws[2] = {1. - us, us};
    T = mub = muq = mus = p = 0.;
    for (int je = 0; je < 2; je++)
      for (int jb = 0; jb < 2; jb++)
        for (int jq = 0; jq < 2; jq++)
          for (int js = 0; js < 2; js++) {
            const size_t k = index(ie + je, ib + jb, iq + jq, is + js);
            const double w = we[je] * wb[jb] * wq[jq] * ws[js];
            p += w * p_[k];
            T += w * T_[k];
            mub += w * mub_[k];
            muq += w * muq_[k];
            mus += w * mus_[k];
          }
    if (p < 0.) p = 0.;
  }
  vh_eos descriptor() const override {
    vh_eos d{};
    d.kind = VH_EOS_TABLE3;
    d.ne = ne_;
    d.nn = nn_;
    d.egrid = eg_.data();
    d.ngrid = ng_.data();
    d.p = p_.data();
    d.T = T_.data();
    d.mub = mub_.data();
    d.muq = muq_.data();
    d.mus = mus_.data();
    return d;
  }
};

// EoSHadron (src/eoHadron.cpp): the hadronic EoS the reference driver gives
// the freeze-out surface (eosTypeHadron 0, src/main.cpp:305-307).  Reads the
// reference's file (header ne nnb nnq e0 n0 logemin logemax lognmax, then
// e nb nq p T mub muq mus status rows, inq fastest) and checks its ranges as
// the constructor does (an exception in place of exit).  As a Fluid's eosH
// it becomes the device's surface EoS (vh_set_surface_eos).
class EoSHadron : public EoS {
  int ne_ = 0, nnb_ = 0, nnq_ = 0;
  double e0_ = 0, n0_ = 0, logemin_ = 0, logemax_ = 0, lognmax_ = 0;
  double nb_abs_min_ = 0, nq_abs_min_ = 0, e_min_ = 0;
  std::vector<double> p_, T_, mub_, muq_, mus_;
  std::vector<int> status_;
  size_t ix3(int ie, int inb, int inq) const {
    return inq + (size_t)nnq_ * inb + (size_t)nnq_ * nnb_ * ie;
  }
  // the position of a charge on the table (src/eoHadron.cpp:97-112)
  static double xpos(double n, double n0, double lognmax, double dxn, double n_abs_min) {
    if (n == 0.0) return 0.;
    const double zn = std::log(std::fabs(n) / n0);
    if (zn >= -lognmax + 2.0 * dxn) return n / std::fabs(n) * 0.5 * (zn + lognmax);
    return n / n_abs_min * dxn;
  }

 public:
  explicit EoSHadron(const char* filename) {
    std::ifstream fin(filename);
    if (!fin) throw Error(VH_ERR_ARG, std::string("EoSHadron: I/O error with ") + filename);
    fin >> ne_ >> nnb_ >> nnq_ >> e0_ >> n0_ >> logemin_ >> logemax_ >> lognmax_;
    if (!fin || ne_ < 2 || nnb_ < 2 || nnq_ < 2) throw Error(VH_ERR_ARG, "EoSHadron: bad header");
    const size_t n = (size_t)ne_ * nnb_ * nnq_;
    for (auto* t : {&p_, &T_, &mub_, &muq_, &mus_}) t->resize(n);
    status_.resize(n);
    std::vector<double> e(ne_), nb(nnb_), nq(nnq_);
    for (int ie = 0; ie < ne_; ie++)
      for (int inb = 0; inb < nnb_; inb++)
        for (int inq = 0; inq < nnq_; inq++) {
          const size_t k = ix3(ie, inb, inq);
          fin >> e[ie] >> nb[inb] >> nq[inq] >> p_[k] >> T_[k] >> mub_[k] >> muq_[k] >> mus_[k] >>
              status_[k];
        }
    if (!fin) throw Error(VH_ERR_ARG, "EoSHadron: truncated table");
    const double dxnb = (2.0 * lognmax_) / (nnb_ - 1), dxnq = (2.0 * lognmax_) / (nnq_ - 1);
    nb_abs_min_ = n0_ * std::exp(2.0 * dxnb - lognmax_);
    nq_abs_min_ = n0_ * std::exp(2.0 * dxnq - lognmax_);
    e_min_ = e0_ * std::exp(logemin_);
    if (std::fabs((e0_ * std::exp(logemin_) - e[0]) / e[0]) > 1e-5 ||
        std::fabs((e0_ * std::exp(logemax_) - e[ne_ - 1]) / e[ne_ - 1]) > 1e-5 ||
        std::fabs(n0_ * std::exp(lognmax_) - nb[nnb_ - 1]) > 1e-4)
      throw Error(VH_ERR_ARG, "EoSHadron: wrong eps or nb range");
  }
  void eos(double e, double nb, double nq, double, double& T, double& mub, double& muq,
           double& mus, double& p) const override {
    T = mub = muq = mus = p = 0.;
    if (e <= 0.) return;
    if (e < e_min_) {
      p = e / e_min_ * p_[ix3(0, nnb_ / 2, nnq_ / 2)];
      T = e / e_min_ * T_[ix3(0, nnb_ / 2, nnq_ / 2)];
      return;
    }
    const double xe = std::log(e / e0_);
    const double dxe = (logemax_ - logemin_) / (ne_ - 1);
    const double dxnb = (2.0 * lognmax_) / (nnb_ - 1), dxnq = (2.0 * lognmax_) / (nnq_ - 1);
    const double xnb = xpos(nb, n0_, lognmax_, dxnb, nb_abs_min_);
    const double xnq = xpos(nq, n0_, lognmax_, dxnq, nq_abs_min_);
    int ie = (int)((xe - logemin_) / dxe), inb = (int)((xnb + lognmax_) / dxnb),
        inq = (int)((xnq + lognmax_) / dxnq);
    ie = std::min(std::max(ie, 0), ne_ - 2);
    inb = std::min(std::max(inb, 0), nnb_ - 2);
    inq = std::min(std::max(inq, 0), nnq_ - 2);
    const double em = xe - logemin_ - ie * dxe, nbm = xnb + lognmax_ - inb * dxnb,
                 nqm = xnq + lognmax_ - inq * dxnq;
    if (status_[ix3(ie, inb, inq)] == 1) return;
    const double we[2] = {1. - em / dxe, em / dxe}, wnb[2] = {1. - nbm / dxnb, nbm / dxnb},
                 wnq[2] = {1. - nqm / dxnq, nqm / dxnq};
    for (int je = 0; je < 2; je++)
      for (int jnb = 0; jnb < 2; jnb++)
        for (int jnq = 0; jnq < 2; jnq++) {
          const size_t k = ix3(ie + je, inb + jnb, inq + jnq);
          p += we[je] * wnb[jnb] * wnq[jnq] * p_[k];
          T += we[je] * wnb[jnb] * wnq[jnq] * T_[k];
          mub += we[je] * wnb[jnb] * wnq[jnq] * mub_[k];
          muq += we[je] * wnb[jnb] * wnq[jnq] * muq_[k];
          mus += we[je] * wnb[jnb] * wnq[jnq] * mus_[k];
        }
    if (p < 0.0) p = 0.0;
  }
  vh_eos descriptor() const override {
    vh_eos d{};
    d.kind = VH_EOS_HADRON;
    d.hadron = vh_eos::vh_eos_hadron{ne_,        nnb_,        nnq_,       e0_,        n0_,
                                     logemin_,   logemax_,    lognmax_,   p_.data(),  T_.data(),
                                     mub_.data(), muq_.data(), mus_.data(), status_.data()};
    return d;
  }
};

// EoSSmash (src/eoSmash.cpp): the SMASH hadron-gas EoS the reference driver
// gives the freeze-out surface for eosTypeHadron 1 (src/main.cpp:308-309,
// eos/hadgas_eos_SMASH.dat with 101 x 51 x 51 points).  Reads the table (a
// header line, then "e nb nq T p muB muS muQ" rows, ie outer, inq inner);
// the grids are uniform from the first to the last row's e, nb, nq, and the
// lookup is trilinear; the device evaluates the same table.
class EoSSmash : public EoS {
  int ne_ = 0, nnb_ = 0, nnq_ = 0;
  double emin_ = 0, emax_ = 0, nbmin_ = 0, nbmax_ = 0, nqmin_ = 0, nqmax_ = 0;
  std::vector<double> p_, T_, mub_, muq_, mus_;
  size_t ix3(int ie, int inb, int inq) const {
    return inq + (size_t)nnq_ * inb + (size_t)nnq_ * nnb_ * ie;
  }

 public:
  EoSSmash(const char* filename, int ne, int nnb, int nnq) : ne_(ne), nnb_(nnb), nnq_(nnq) {
    std::ifstream fin(filename);
    if (!fin) throw Error(VH_ERR_ARG, std::string("EoSSmash: I/O error with ") + filename);
    if (ne < 2 || nnb < 2 || nnq < 2) throw Error(VH_ERR_ARG, "EoSSmash: bad table dimensions");
    std::string header;
    std::getline(fin, header);
    const size_t n = (size_t)ne_ * nnb_ * nnq_;
    for (auto* t : {&p_, &T_, &mub_, &muq_, &mus_}) t->resize(n);
    double e = 0, nb = 0, nq = 0;
    for (int ie = 0; ie < ne_; ie++)
      for (int inb = 0; inb < nnb_; inb++)
        for (int inq = 0; inq < nnq_; inq++) {
          const size_t k = ix3(ie, inb, inq);
          fin >> e >> nb >> nq >> T_[k] >> p_[k] >> mub_[k] >> mus_[k] >> muq_[k];
          if (k == 0) {
            emin_ = e;
            nbmin_ = nb;
            nqmin_ = nq;
          }
        }
    if (!fin) throw Error(VH_ERR_ARG, "EoSSmash: truncated table");
    emax_ = e;
    nbmax_ = nb;
    nqmax_ = nq;
    if (!(emin_ < emax_) || !(nbmin_ < nbmax_) || !(nqmin_ < nqmax_))
      throw Error(VH_ERR_ARG, "EoSSmash: the table's e, nb, nq ranges are empty");
  }
  void eos(double e, double nb, double nq, double, double& T, double& mub, double& muq,
           double& mus, double& p) const override {
    T = mub = muq = mus = p = 0.;
    if (e <= 0.) return;
    if (e < emin_) {
      p = e / emin_ * p_[ix3(0, nnb_ / 2, nnq_ / 2)];
      T = e / emin_ * T_[ix3(0, nnb_ / 2, nnq_ / 2)];
      return;
    }
    const double de = (emax_ - emin_) / (ne_ - 1), dnb = (nbmax_ - nbmin_) / (nnb_ - 1),
                 dnq = (nqmax_ - nqmin_) / (nnq_ - 1);
    int ie = (int)((e - emin_) / de), inb = (int)((nb - nbmin_) / dnb),
        inq = (int)((nq - nqmin_) / dnq);
    ie = std::min(std::max(ie, 0), ne_ - 2);
    inb = std::min(std::max(inb, 0), nnb_ - 2);
    inq = std::min(std::max(inq, 0), nnq_ - 2);
    const double em = e - emin_ - ie * de, nbm = nb - nbmin_ - inb * dnb,
                 nqm = nq - nqmin_ - inq * dnq;
    const double we[2] = {1. - em / de, em / de}, wnb[2] = {1. - nbm / dnb, nbm / dnb},
                 wnq[2] = {1. - nqm / dnq, nqm / dnq};
    for (int je = 0; je < 2; je++)
      for (int jnb = 0; jnb < 2; jnb++)
        for (int jnq = 0; jnq < 2; jnq++) {
          const size_t k = ix3(ie + je, inb + jnb, inq + jnq);
          const double w = we[je] * wnb[jnb] * wnq[jnq];
          p += w * p_[k];
          T += w * T_[k];
          mub += w * mub_[k];
          muq += w * muq_[k];
          mus += w * mus_[k];
        }
    if (p < 0.0) p = 0.0;
  }
  vh_eos descriptor() const override {
    vh_eos d{};
    d.kind = VH_EOS_SMASH;
    d.smash = vh_eos::vh_eos_smash{ne_,    nnb_,   nnq_,      emin_,     emax_,
                                   nbmin_, nbmax_, nqmin_,    nqmax_,    p_.data(),
                                   T_.data(), mub_.data(), muq_.data(), mus_.data()};
    return d;
  }
};

// EoSAZH (src/eoAZH.cpp): the reference driver's eosType 2.  Reads
// dir/eos/azhydro0p2/aa{1,2}_{p,t,mb}.dat in the EoSAZHaux format (header
// "nmin emin", "dn de nn ne" with one point fewer than stored on each axis,
// then the values with e outer); p, T and muB come from the first table set
// inside its e range, from the second above it and from the first set's
// first row scaled by e / emin below it; the device evaluates the same tables.
class EoSAZH : public EoS {
  struct Tab {
    int ne = 0, nn = 0;
    double emin = 0, nmin = 0, de = 0, dn = 0;
    std::vector<double> v;  // [ie * nn + in]
    explicit Tab(const std::string& path) {
      std::ifstream fin(path);
      if (!fin.good()) throw Error(VH_ERR_ARG, "EoSAZH: I/O error with " + path);
      fin >> nmin >> emin >> dn >> de >> nn >> ne;
      nn++;
      ne++;
      if (!fin || ne < 2 || nn < 2 || !(de > 0.) || !(dn > 0.) || !(emin > 0.))
        throw Error(VH_ERR_ARG, "EoSAZH: bad header in " + path);
      v.resize((size_t)ne * nn);
      for (double& x : v) fin >> x;
      if (!fin) throw Error(VH_ERR_ARG, "EoSAZH: truncated table " + path);
    }
    double get(double e, double nb) const {  // EoSAZHaux::get
      if (e <= 0.) return 0.0;
      int ie = (int)((e - emin) / de), in = (int)((nb - nmin) / dn);
      ie = std::min(std::max(ie, 0), ne - 2);
      in = std::min(std::max(in, 0), nn - 2);
      const double em = (e - emin - ie * de) / de, nm = (nb - nmin - in * dn) / dn;
      const double we[2] = {1. - em, em}, wn[2] = {1. - nm, nm};
      double value = 0.0;
      for (int je = 0; je < 2; je++)
        for (int jn = 0; jn < 2; jn++) value += we[je] * wn[jn] * v[(size_t)(ie + je) * nn + in + jn];
      return value;
    }
    double getLow(double e, double nb) const {  // EoSAZHaux::getLow
      if (e <= 0.) return 0.0;
      int in = (int)((nb - nmin) / dn);
      in = std::min(std::max(in, 0), nn - 2);
      const double nm = (nb - nmin - in * dn) / dn;
      const double value = (1. - nm) * v[in] + nm * v[in + 1];
      return value * e / emin;
    }
    vh_eos::vh_eos_azh::vh_eos_azh_table desc() const {
      return {ne, nn, emin, nmin, de, dn, v.data()};
    }
  };
  std::vector<Tab> t_;  // p1, p2, T1, T2, mu1, mu2

 public:
  explicit EoSAZH(const std::string& dir) {
    for (const char* f : {"aa1_p", "aa2_p", "aa1_t", "aa2_t", "aa1_mb", "aa2_mb"})
      t_.emplace_back(dir + "/eos/azhydro0p2/" + f + ".dat");
  }
  void eos(double e, double nb, double, double, double& T, double& mub, double& muq,
           double& mus, double& p) const override {
    const double anb = std::fabs(nb);
    const Tab& p1 = t_[0];
    if (e > p1.emin + p1.de * (p1.ne - 1)) {
      p = t_[1].get(e, anb);
      T = t_[3].get(e, anb);
      mub = t_[5].get(e, nb);
    } else if (e > p1.emin) {
      p = t_[0].get(e, anb);
      T = t_[2].get(e, anb);
      mub = t_[4].get(e, nb);
    } else {
      p = t_[0].getLow(e, anb);
      T = t_[2].getLow(e, anb);
      mub = t_[4].getLow(e, nb);
    }
    muq = mus = 0.0;
  }
  vh_eos descriptor() const override {
    vh_eos d{};
    d.kind = VH_EOS_AZH;
    d.azh = {t_[0].desc(), t_[1].desc(), t_[2].desc(), t_[3].desc(), t_[4].desc(), t_[5].desc()};
    return d;
  }
};

// EoSCMFe (src/eoCMFe.cpp): the reference driver's eosType 4.  Reads
// dir/eos/cmfe_small.dat (1501 x 501) and dir/eos/cmfe.dat (4001 x 401): a
// header line, then e n T p s muB muS rows with e outer (NAN allowed),
// converted to GeV/fm^3, fm^-3 and GeV as its constructor does; the
// lookup is EoSChiral's with a cutoff at e = 2e-2 and a NaN pressure
// replaced; the device evaluates the same tables.
class EoSCMFe : public EoS {
  static constexpr double kEps0 = 146.51751415742 * 0.87326281;
  static constexpr double kN0 = 0.15891 * 0.87272727;
  struct Aux {
    int ne, nn;
    double emin = 0., emax = 0., nmin = 0., nmax = 0.;
    std::vector<double> p, T, mub, mus;  // [in * ne + ie]
    Aux(const std::string& path, int Ne, int Nn) : ne(Ne), nn(Nn) {
      std::ifstream fin(path);
      if (!fin.good()) throw Error(VH_ERR_ARG, "EoSCMFe: I/O error with " + path);
      fin.ignore(1000, '\n');
      const size_t n = (size_t)ne * nn;
      for (auto* t : {&p, &T, &mub, &mus}) t->resize(n);
      auto num = [&fin]() {
        std::string w;
        fin >> w;
        return w == "NAN" ? std::numeric_limits<double>::quiet_NaN() : std::atof(w.c_str());
      };
      double e0 = 0., e1 = 0., n0 = 0., n1 = 0.;
      for (int ie = 0; ie < ne; ie++)
        for (int in = 0; in < nn; in++) {
          const size_t k = (size_t)in * ne + ie;
          const double e = num() * kEps0 / 1000.0, nb = num() * kN0;
          T[k] = num() / 1000.0;
          p[k] = num() * kEps0 / 1000.0;
          num();  // s
          mub[k] = num() / 1000.0;
          mus[k] = num() / 1000.0;
          if (ie == 0) e0 = e;
          if (ie == ne - 1) e1 = e;
          if (in == 0) n0 = nb;
          if (in == nn - 1) n1 = nb;
        }
      if (!fin) throw Error(VH_ERR_ARG, "EoSCMFe: truncated table " + path);
      emin = e0;
      emax = e1;
      nmin = n0;
      nmax = n1;
    }
    void get(double e, double nb, double& pp, double& TT, double& mb, double& ms) const {
      if (e < 2e-2) {
        TT = mb = ms = pp = 0.;
        return;
      }
      const double de = (emax - emin) / (ne - 1), dn = (nmax - nmin) / (nn - 1);
      int ie = (int)((e - emin) / de), in = (int)((nb - nmin) / dn);
      ie = std::min(std::max(ie, 0), ne - 2);
      in = std::min(std::max(in, 0), nn - 2);
      const double em = e - emin - ie * de, nm = nb - nmin - in * dn;
      const double we[2] = {1. - em / de, em / de}, wn[2] = {1. - nm / dn, nm / dn};
      TT = mb = ms = pp = 0.0;
      for (int je = 0; je < 2; je++)
        for (int jn = 0; jn < 2; jn++) {
          const size_t k = (size_t)(in + jn) * ne + (ie + je);
          pp += we[je] * wn[jn] * p[k];
          TT += we[je] * wn[jn] * T[k];
          mb += we[je] * wn[jn] * mub[k];
          ms += we[je] * wn[jn] * mus[k];
        }
      if (std::isnan(pp)) {
        if (e > 0.8 * kEps0 || nb > 40. * kN0) {
          pp = 0.2964 * e;
          TT = 0.15120476935 * std::pow(e, 0.25);
          mb = ms = 0.0;
        } else {
          TT = mb = ms = pp = 0.;
        }
      }
      if (pp < 0.0) pp = 0.0;
    }
    vh_eos_aux desc() const {
      return {ne, nn, emin, emax, nmin, nmax, p.data(), T.data(), mub.data(), mus.data()};
    }
  };
  Aux small_, big_;

 public:
  explicit EoSCMFe(const std::string& dir)
      : small_(dir + "/eos/cmfe_small.dat", 1501, 501), big_(dir + "/eos/cmfe.dat", 4001, 401) {}
  void eos(double e, double nb, double, double, double& T, double& mub, double& muq,
           double& mus, double& p) const override {
    if (e < 15 * kEps0 / 1000.0 && nb < 5 * kN0)
      small_.get(e, nb, p, T, mub, mus);
    else if (e < 0.8 * kEps0 && nb < 40. * kN0)
      big_.get(e, nb, p, T, mub, mus);
    else {
      p = 0.2964 * e;
      T = 0.15120476935 * std::pow(e, 0.25);
      mub = mus = 0.0;
    }
    muq = 0.0;
  }
  vh_eos descriptor() const override {
    vh_eos d{};
    d.kind = VH_EOS_CMFE;
    d.aux[0] = small_.desc();
    d.aux[1] = big_.desc();
    return d;
  }
};

// EoSChiral (src/eoChiral.cpp): the reference's default EoS (eosType 1).
// Reads dir/eos/chiraleos.dat (2001 x 401) and dir/eos/chiralsmall.dat
// (201 x 201) in the EoSaux format (8 columns, nb outer, e inner) with its
// unit conversions; the device evaluates the same tables.
class EoSChiral : public EoS {
  struct Aux {
    int ne, nn;
    double emin = 0., emax = 0., nmin = 0., nmax = 0.;
    std::vector<double> p, T, mub, mus;  // [in * ne + ie]
    Aux(const std::string& path, int Ne, int Nn) : ne(Ne), nn(Nn) {
      std::ifstream fin(path);
      if (!fin.good()) throw Error(VH_ERR_ARG, "EoSChiral: I/O error with " + path);
      const size_t n = (size_t)ne * nn;
      p.resize(n);
      T.resize(n);
      mub.resize(n);
      mus.resize(n);
      std::vector<double> e(ne), nb(nn);
      double s, a;
      for (int in = 0; in < nn; in++)
        for (int ie = 0; ie < ne; ie++) {
          const size_t k = (size_t)in * ne + ie;
          fin >> T[k] >> mub[k] >> e[ie] >> p[k] >> nb[in] >> s >> mus[k] >> a;
          T[k] /= 1000.0;
          mub[k] *= 3.0 / 1000.0;
          mus[k] /= 1000.0;
          p[k] *= 0.146;
        }
      if (!fin) throw Error(VH_ERR_ARG, "EoSChiral: truncated table " + path);
      emin = e[0] * 0.146;
      emax = e[ne - 1] * 0.146;
      nmin = nb[0] * 0.15;
      nmax = nb[nn - 1] * 0.15;
    }
    void get(double e, double n, double& pp, double& TT, double& mb, double& ms) const {
      if (e < 0.) {
        TT = mb = ms = pp = 0.;
        return;
      }
      const double de = (emax - emin) / (ne - 1), dn = (nmax - nmin) / (nn - 1);
      int ie = (int)((e - emin) / de), in = (int)((n - nmin) / dn);
      ie = std::min(std::max(ie, 0), ne - 2);
      in = std::min(std::max(in, 0), nn - 2);
      const double em = e - emin - ie * de, nm = n - nmin - in * dn;
      const double we[2] = {1. - em / de, em / de}, wn[2] = {1. - nm / dn, nm / dn};
      TT = mb = ms = pp = 0.0;
      for (int je = 0; je < 2; je++)
        for (int jn = 0; jn < 2; jn++) {
          const size_t k = (size_t)(in + jn) * ne + ie + je;
          pp += we[je] * wn[jn] * p[k];
          TT += we[je] * wn[jn] * T[k];
          mb += we[je] * wn[jn] * mub[k];
          ms += we[je] * wn[jn] * mus[k];
        }
      if (pp < 0.0) pp = 0.0;
    }
    vh_eos_aux view() const {
      return vh_eos_aux{ne, nn, emin, emax, nmin, nmax, p.data(), T.data(), mub.data(), mus.data()};
    }
  };
  Aux small_, big_;

 public:
  explicit EoSChiral(const std::string& dir = ".")
      : small_(dir + "/eos/chiralsmall.dat", 201, 201), big_(dir + "/eos/chiraleos.dat", 2001, 401) {}
  void eos(double e, double nb, double, double, double& T, double& mub, double& muq,
           double& mus, double& p) const override {
    if (e < 1.46 && nb < 0.3)
      small_.get(e, nb, p, T, mub, mus);
    else if (e < 146. && nb < 6.)
      big_.get(e, nb, p, T, mub, mus);
    else {
      p = 0.2964 * e;
      T = 0.15120476935 * std::pow(e, 0.25);
      mub = mus = 0.0;
    }
    muq = 0.0;
  }
  vh_eos descriptor() const override {
    vh_eos d{};
    d.kind = VH_EOS_CHIRAL;
    d.aux[0] = small_.view();
    d.aux[1] = big_.view();
    return d;
  }
};

// -------------------------------------------------------- TransportCoeff
// src/trancoeff.h:6-45: the same public constants and constructor.
class TransportCoeff {
 public:
  const double etaS0, zetaS0, ah, al, aRho, T0, etaSMin, etaSEpsilonMin, etaSShiftMuB,
      etaSScaleMuB, zetaSPeakEpsilon, zetaSScaleBeta, zetaSSigmaMinus, zetaSSigmaPlus;
  EoS* eos;
  const int etaSparam, zetaSparam;
  // zetaSparam 5 (a Gaussian bump in T; not in the reference)
  double zetaSPeakT = 0.175, zetaSWidthT = 0.02;
  TransportCoeff(double _etaS0, double _zetaS0, double _ah, double _al, double _aRho, double _T0,
                 double _etaSMin, double _etaSEpsilonMin, double _etaSShiftMuB,
                 double _etaSScaleMuB, double _zetaSPeakEpsilon, double _zetaSScaleBeta,
                 double _zetaSSigmaMinus, double _zetaSSigmaPlus, EoS* _eos, int _etaSparam,
                 int _zetaSparam)
      : etaS0(_etaS0), zetaS0(_zetaS0), ah(_ah), al(_al), aRho(_aRho), T0(_T0),
        etaSMin(_etaSMin), etaSEpsilonMin(_etaSEpsilonMin), etaSShiftMuB(_etaSShiftMuB),
        etaSScaleMuB(_etaSScaleMuB), zetaSPeakEpsilon(_zetaSPeakEpsilon),
        zetaSScaleBeta(_zetaSScaleBeta), zetaSSigmaMinus(_zetaSSigmaMinus),
        zetaSSigmaPlus(_zetaSSigmaPlus), eos(_eos), etaSparam(_etaSparam),
        zetaSparam(_zetaSparam) {}
  bool isViscous() const {
    return etaS0 > 0. || zetaS0 > 0. || etaSparam > 0 || zetaSparam > 0;
  }
  vh_trcoeff descriptor() const {
    return vh_trcoeff{etaS0,         zetaS0,         ah,           al,
                      aRho,          T0,             etaSMin,      etaSEpsilonMin,
                      etaSShiftMuB,  etaSScaleMuB,   zetaSPeakEpsilon, zetaSScaleBeta,
                      zetaSSigmaMinus, zetaSSigmaPlus, etaSparam,   zetaSparam,
                      zetaSPeakT,      zetaSWidthT};
  }
};

// ------------------------------------------------------------------ Fluid
// src/fld.h: the grid and a host copy of every cell (structure of arrays).
class Fluid {
  EoS *eos_, *eosH_;
  TransportCoeff* tr_;
  int nx_, ny_, nz_;
  double minx_, maxx_, miny_, maxy_, minz_, maxz_, dx_, dy_, dz_, dt_, ecrit_;
  long long N_;

 public:
  std::vector<double> Q, Qh, Qprev, pi, piH, Pi, PiH, m, vcc;

  EoS* eos() const { return eos_; }
  EoS* eosH() const { return eosH_; }
  Fluid(EoS* eos, EoS* eosH, TransportCoeff* tr, int nx, int ny, int nz, double minx,
        double maxx, double miny, double maxy, double minz, double maxz, double dt, double eCrit)
      : eos_(eos), eosH_(eosH), tr_(tr), nx_(nx), ny_(ny), nz_(nz), minx_(minx), maxx_(maxx),
        miny_(miny), maxy_(maxy), minz_(minz), maxz_(maxz), dt_(dt), ecrit_(eCrit) {
    dx_ = (maxx - minx) / (nx - 1);  // src/fld.cpp:77-79
    dy_ = (maxy - miny) / (ny - 1);
    dz_ = (maxz - minz) / (nz - 1);
    N_ = (long long)nx * ny * nz;
    Q.assign(7 * N_, 0.);
    Qh.assign(7 * N_, 0.);
    Qprev.assign(7 * N_, 0.);
    pi.assign(10 * N_, 0.);
    piH.assign(10 * N_, 0.);
    Pi.assign(N_, 0.);
    PiH.assign(N_, 0.);
    m.assign(3 * N_, 0.);
    vcc.assign(N_, 1.);
  }
  int getNX() const { return nx_; }
  int getNY() const { return ny_; }
  int getNZ() const { return nz_; }
  double getDx() const { return dx_; }
  double getDy() const { return dy_; }
  double getDz() const { return dz_; }
  double getX(int ix) const { return minx_ + ix * dx_; }
  double getY(int iy) const { return miny_ + iy * dy_; }
  double getZ(int iz) const { return minz_ + iz * dz_; }
  double geteCrit() const { return ecrit_; }
  EoS* getEoS() const { return eos_; }
  long long ncells() const { return N_; }
  vh_grid grid() const { return vh_grid{nx_, ny_, nz_, minx_, maxx_, miny_, maxy_, minz_, maxz_, 0.}; }
  // Fluid::getCell clamping (src/fld.h:70-78)
  long long index(int ix, int iy, int iz) const {
    ix = std::min(std::max(ix, 0), nx_ - 1);
    iy = std::min(std::max(iy, 0), ny_ - 1);
    iz = std::min(std::max(iz, 0), nz_ - 1);
    return ix + (long long)nx_ * iy + (long long)nx_ * ny_ * iz;
  }
  // Cell accessors (src/cll.h)
  void getQ(int ix, int iy, int iz, double* q) const {
    const long long i = index(ix, iy, iz);
    for (int k = 0; k < 7; k++) q[k] = Q[k * N_ + i];
  }
  void setQ(int ix, int iy, int iz, const double* q) {  // Cell::setQ zeroing, src/cll.h:75-80
    const long long i = index(ix, iy, iz);
    const bool neg = q[T_] < 0.;
    for (int k = 0; k < 7; k++) Q[k * N_ + i] = neg ? 0. : q[k];
  }
  void saveQprev(int ix, int iy, int iz) {
    const long long i = index(ix, iy, iz);
    for (int k = 0; k < 7; k++) Qprev[k * N_ + i] = Q[k * N_ + i];
  }
  void setAllM(int ix, int iy, int iz, double v) {
    const long long i = index(ix, iy, iz);
    for (int d = 0; d < 3; d++) m[d * N_ + i] = v;
  }
  double getM(int ix, int iy, int iz, int dir) const { return m[(dir - 1) * N_ + index(ix, iy, iz)]; }
  double getpi(int ix, int iy, int iz, int a, int b) const {
    return pi[index44(a, b) * N_ + index(ix, iy, iz)];
  }
  double getPi(int ix, int iy, int iz) const { return Pi[index(ix, iy, iz)]; }
  double getViscCorrCutFlag(int ix, int iy, int iz) const { return vcc[index(ix, iy, iz)]; }
  // Cell::setPrimVar, src/cll.cpp:222-241
  void setPrimVar(int ix, int iy, int iz, double tau, double e, double nb, double nq, double ns,
                  double vx, double vy, double vz) {
    const double gamma2 = 1. / (1 - vx * vx - vy * vy - vz * vz);
    const double p = eos_->p(e, nb, nq, ns);
    double q[7];
    q[T_] = tau * (e + p * (vx * vx + vy * vy + vz * vz)) * gamma2;
    q[X_] = tau * (e + p) * vx * gamma2;
    q[Y_] = tau * (e + p) * vy * gamma2;
    q[Z_] = tau * (e + p) * vz * gamma2;
    q[NB_] = tau * nb * std::sqrt(gamma2);
    q[NQ_] = tau * nq * std::sqrt(gamma2);
    q[NS_] = tau * ns * std::sqrt(gamma2);
    const long long i = index(ix, iy, iz);
    for (int k = 0; k < 7; k++) Q[k * N_ + i] = q[k];
  }
  vh_state_view view() {
    return vh_state_view{Q.data(), Qh.data(), Qprev.data(), pi.data(), piH.data(),
                         Pi.data(), PiH.data(), m.data(), vcc.data()};
  }

  // Grid snapshot (initial state or checkpoint): 8-byte tag "VHBSNAP1",
  // int32 nx ny nz 0, float64 xmin xmax ymin ymax etamin etamax tau dt, then
  // the planes Q Qh Qprev pi piH Pi PiH m viscCorrCut as raw float64.
  struct SnapshotHeader {
    vh_grid grid;
    double tau, dt;
  };
  static SnapshotHeader readSnapshotHeader(const char* path) {
    std::ifstream in(path, std::ios::binary);
    char tag[8];
    int32_t n[4];
    double b[8];
    in.read(tag, 8);
    in.read(reinterpret_cast<char*>(n), sizeof n);
    in.read(reinterpret_cast<char*>(b), sizeof b);
    if (!in || std::memcmp(tag, "VHBSNAP1", 8) != 0)
      throw Error(VH_ERR_ARG, std::string("not a grid snapshot: ") + path);
    return SnapshotHeader{vh_grid{n[0], n[1], n[2], b[0], b[1], b[2], b[3], b[4], b[5], 0.}, b[6],
                          b[7]};
  }
  void loadSnapshot(const char* path) {
    const SnapshotHeader h = readSnapshotHeader(path);
    if (h.grid.nx != nx_ || h.grid.ny != ny_ || h.grid.nz != nz_)
      throw Error(VH_ERR_ARG, "snapshot grid size differs from the fluid's");
    std::ifstream in(path, std::ios::binary);
    in.seekg(8 + 4 * 4 + 8 * 8);
    for (std::vector<double>* v : planes())
      in.read(reinterpret_cast<char*>(v->data()), (std::streamsize)(v->size() * sizeof(double)));
    if (!in) throw Error(VH_ERR_ARG, std::string("truncated snapshot: ") + path);
  }
  void saveSnapshot(const char* path, double tau, double dt) {
    std::ofstream out(path, std::ios::binary);
    const int32_t n[4] = {nx_, ny_, nz_, 0};
    const double b[8] = {minx_, maxx_, miny_, maxy_, minz_, maxz_, tau, dt};
    out.write("VHBSNAP1", 8);
    out.write(reinterpret_cast<const char*>(n), sizeof n);
    out.write(reinterpret_cast<const char*>(b), sizeof b);
    for (std::vector<double>* v : planes())
      out.write(reinterpret_cast<const char*>(v->data()), (std::streamsize)(v->size() * sizeof(double)));
    if (!out) throw Error(VH_ERR_ARG, std::string("cannot write snapshot: ") + path);
  }

 private:
  std::vector<std::vector<double>*> planes() {
    return {&Q, &Qh, &Qprev, &pi, &piH, &Pi, &PiH, &m, &vcc};
  }
};

// Interior totals printed by Fluid::outputSurface (src/fld.cpp:544-604).
struct Totals {
  double E, Efull, Nb1, Nb2, S, Px, vt_num, vt_den, vxvy_num, vxvy_den, pi0x_num, pi0x_den,
      txxyy_num, txxyy_den, nCoreCells, nCoreCutCells;
};

// ------------------------------------------------------------------ Hydro
// src/hdo.h: one timestep of the whole grid per performStep(), on the GPU.
class Hydro {
  Fluid* f_;
  EoS* eos_;
  TransportCoeff* tr_;
  vh_ctx* ctx_ = nullptr;
  int device_;
  double t0_, dt0_;
  bool uploaded_ = false;
  bool vorticity_ = false;

  void create() {
    const vh_grid g = f_->grid();
    const vh_eos e = eos_->descriptor();
    const vh_trcoeff t = tr_->descriptor();
    check(vh_create(&g, &e, &t, t0_, dt0_, device_, &ctx_), nullptr);
    if (vorticity_) check(vh_enable_vorticity(ctx_, 1), ctx_);  // new cells: zero dbeta
    // the Fluid's eosH is the EoS of outputSurface / outputCorona
    // (src/fld.cpp:540-542, 885-887)
    if (f_->eosH() && f_->eosH() != eos_) {
      const vh_eos h = f_->eosH()->descriptor();
      check(vh_set_surface_eos(ctx_, &h), ctx_);
    }
  }

 public:
  Hydro(Fluid* f, EoS* eos, TransportCoeff* tr, double t0, double dt, int device = 0)
      : f_(f), eos_(eos), tr_(tr), device_(device), t0_(t0), dt0_(dt) {
    create();
  }
  ~Hydro() { vh_destroy(ctx_); }
  Hydro(const Hydro&) = delete;
  Hydro& operator=(const Hydro&) = delete;

  // Hydro::setDtau (src/hdo.cpp:67-75); the reference exits on dt > dx/2.
  void setDtau(double dt) { check(vh_set_dtau(ctx_, dt), ctx_); }
  double getDtau() const {
    double d;
    check(vh_get_dtau(ctx_, &d), ctx_);
    return d;
  }
  double getTau() const {
    double t;
    check(vh_get_tau(ctx_, &t), ctx_);
    return t;
  }
  Fluid* getFluid() const { return f_; }
  // Hydro::setFluid: the new Fluid's cells replace the device grid.
  void setFluid(Fluid* f) {
    const double tau = getTau(), dt = getDtau();
    vh_destroy(ctx_);
    ctx_ = nullptr;
    f_ = f;
    t0_ = tau;
    dt0_ = dt;
    create();
    uploaded_ = false;
  }
  // Copies the Fluid's host cells to the device (done by the first step).
  void upload() {
    vh_state_view v = f_->view();
    check(vh_upload_state(ctx_, &v), ctx_);
    uploaded_ = true;
  }
  // Hydro::performStep (src/hdo.cpp:1016-1134)
  void performStep() {
    if (!uploaded_) upload();
    check(vh_step(ctx_), ctx_);
  }
  // Waits for the device and copies every cell back into the Fluid.
  void sync() {
    check(vh_sync(ctx_), ctx_);
    vh_state_view v = f_->view();
    check(vh_download_state(ctx_, &v), ctx_);
  }
  Totals totals() {
    Totals t;
    check(vh_totals(ctx_, f_->geteCrit(), &t.E), ctx_);
    return t;
  }
  // The freeze-out elements of Fluid::outputSurface (src/fld.cpp:606-842)
  // at the current tau, kept on the device; writeSurface appends them to a
  // freezeout.dat-format file (extended records with e and nb if asked).
  vh_surface_info surface() {
    vh_surface_info si{};
    check(vh_surface(ctx_, f_->geteCrit(), &si), ctx_);
    return si;
  }
  // The corona of Fluid::outputCorona (src/fld.cpp:876-1089) at the current
  // tau (the reference driver writes it once at tau0); writeSurface then
  // appends its records.
  vh_surface_info corona() {
    if (!uploaded_) upload();
    vh_surface_info si{};
    check(vh_corona(ctx_, f_->geteCrit(), &si), ctx_);
    return si;
  }
  void writeSurface(const char* path, bool extendFO) {
    check(vh_surface_write(ctx_, path, extendFO ? 1 : 0), ctx_);
  }
  // Hydro::enableVorticity (src/hdo.cpp:60-64): every later viscous step
  // stores d_mu beta_nu per cell, and surface() computes the beta.dat values.
  void enableVorticity() {
    vorticity_ = true;
    check(vh_enable_vorticity(ctx_, 1), ctx_);
  }
  // Cell::getDbeta of every cell: out[(4 mu + nu) * N + i] (16 N doubles).
  void getDbeta(double* out) { check(vh_get_dbeta(ctx_, out), ctx_); }
  // Appends the last surface() call's beta.dat lines to `path`; with header,
  // Fluid::printDbetaHeader's lines first (after corona(), src/main.cpp:391).
  void writeBeta(const char* path, bool header) {
    check(vh_surface_write_beta(ctx_, path, header ? 1 : 0), ctx_);
  }
  // The driver's substep block (src/main.cpp:405-419); returns the count.
  int advance(double dtau, double etamin, double etamax, int nz) {
    if (!uploaded_) upload();
    int n = 1;
    check(vh_advance(ctx_, dtau, etamin, etamax, nz, &n), ctx_);
    return n;
  }
  vh_ctx* context() const { return ctx_; }
  // The device cells were set by a device builder (IcGlissando::setIC and
  // the like below): the first step must not upload the host Fluid's.
  void adoptDeviceState() { uploaded_ = true; }

  // expandGrid2x (src/main.cpp:246-271): the device grid doubles its
  // transverse range and the step doubles.  Returns the new host Fluid (its
  // cells are filled by the next sync()) and deletes the old one, or
  // returns the old Fluid when the grid is not symmetric.
  friend Fluid* expandGrid2x(Hydro* h, EoS* eos, EoS* eosH, TransportCoeff* tr);
};

inline Fluid* expandGrid2x(Hydro* h, EoS* eos, EoS* eosH, TransportCoeff* tr) {
  Fluid* f = h->getFluid();
  int resized = 0;
  check(vh_resize2x(h->ctx_, &resized), h->ctx_);
  if (!resized) {
    std::cout << "this grid expansion works only with symmetric min/max ranges\n";
    return f;
  }
  vh_grid g;
  check(vh_get_grid(h->ctx_, &g), h->ctx_);
  Fluid* fnew = new Fluid(eos, eosH, tr, g.nx, g.ny, g.nz, g.xmin, g.xmax, g.ymin, g.ymax,
                          g.etamin, g.etamax, h->getDtau(), f->geteCrit());
  h->f_ = fnew;
  delete f;
  return fnew;
}

// ------------------------------------------------------ initial states
// The reference's IC modules (src/icGlissando.h, src/icTrento.h,
// src/icGubser.h, src/ic.h) with their constructors' file reading, built on
// the device: setIC fills the Hydro's device cells (vh_init_glissando,
// vh_init_trento, vh_init_gubser, vh_init_table) at the Hydro's tau, where
// the reference's setIC(Fluid*, EoS*) fills host cells; call sync() for a
// host copy.  An unknown setup name throws (the reference exits).

// IcGlissando (icModel 5): "x y c w" lines, c != 0 kept, a line that does
// not parse ending an event that holds sources (src/icGlissando.cpp:130-160)
class IcGlissando {
  vh_ic_setup setup_{};
  std::vector<double> x_, y_;
  std::vector<int> c_, npart_;

 public:
  IcGlissando(Fluid*, const char* filename, double /*tau0: the Hydro's*/, const char* setup) {
    check(vh_ic_setup_named(5, setup, &setup_), nullptr);
    std::ifstream fin(filename);
    if (!fin.good()) throw Error(VH_ERR_ARG, std::string("I/O error with ") + filename);
    std::string line;
    int np = 0;
    // line by line until end of file: a file that ends with a newline gives
    // a last, empty line, which ends the last event (without the newline the
    // last event is not counted, as in the reference)
    while (!fin.eof()) {
      std::getline(fin, line);
      std::istringstream in(line);
      double x, y, w;
      int c;
      if (in >> x >> y >> c >> w) {
        if (c != 0) {
          x_.push_back(x);
          y_.push_back(y);
          c_.push_back(c);
          if (++np > 9999) throw Error(VH_ERR_ARG, "IcGlissando: more sources in an event than NP");
        }
      } else if (np > 0) {
        npart_.push_back(np);
        np = 0;
      }
    }
    if (npart_.empty()) throw Error(VH_ERR_ARG, std::string("no GLISSANDO events in ") + filename);
  }
  int nevents() const { return (int)npart_.size(); }
  const std::vector<double>& x() const { return x_; }
  const std::vector<double>& y() const { return y_; }
  const std::vector<int>& c() const { return c_; }
  const std::vector<int>& npart() const { return npart_; }
  // returns sNorm, nNorm
  std::pair<double, double> setIC(Hydro* h) {
    vh_glissando_ic ic{setup_, x_.data(), y_.data(), c_.data(), npart_.data(), nevents()};
    double norms[2];
    check(vh_init_glissando(h->context(), &ic, norms), h->context());
    h->adoptDeviceState();
    return {norms[0], norms[1]};
  }
};

// IcTrento (icModel 7): per event the header's npart (line 3, column 9),
// grid-nsteps (line 10, column 15) and grid-max (line 11, column 12), then
// n rows of n values; an empty third header line ends the file
// (src/icTrento.cpp:115-179)
class IcTrento {
  vh_ic_setup setup_{};
  std::vector<double> grid_, gmax_;
  std::vector<int> ngrid_, npart_;

 public:
  IcTrento(Fluid*, const char* filename, double /*tau0: the Hydro's*/, const char* setup) {
    check(vh_ic_setup_named(7, setup, &setup_), nullptr);
    std::ifstream fin(filename);
    if (!fin.good()) throw Error(VH_ERR_ARG, std::string("I/O error with ") + filename);
    auto field = [](const std::string& l, size_t col) {
      return l.size() > col ? l.substr(col) : std::string();
    };
    for (;;) {
      std::string l[11];
      for (int k = 0; k < 3; k++) std::getline(fin, l[k]);
      if (l[2].empty()) break;
      for (int k = 3; k < 11; k++) std::getline(fin, l[k]);
      int npart = 0, n = 0;
      double gmax = 0.;
      std::istringstream(field(l[2], 9)) >> npart;
      std::istringstream(field(l[9], 15)) >> n;
      std::istringstream(field(l[10], 12)) >> gmax;
      if (n < 2) throw Error(VH_ERR_ARG, std::string("bad grid-nsteps in ") + filename);
      for (long long k = 0; k < (long long)n * n; k++) {
        double v = 0.;
        fin >> v;
        grid_.push_back(v);
      }
      std::string rest;
      std::getline(fin, rest);
      npart_.push_back(npart);
      ngrid_.push_back(n);
      gmax_.push_back(gmax);
    }
    if (npart_.empty()) throw Error(VH_ERR_ARG, std::string("no TRENTO events in ") + filename);
  }
  int nevents() const { return (int)npart_.size(); }
  const std::vector<double>& grid() const { return grid_; }
  const std::vector<int>& ngrid() const { return ngrid_; }
  const std::vector<double>& gmax() const { return gmax_; }
  const std::vector<int>& npart() const { return npart_; }
  std::pair<double, double> setIC(Hydro* h) {
    vh_trento_ic ic{setup_, grid_.data(), ngrid_.data(), gmax_.data(), npart_.data(), nevents()};
    double norms[2];
    check(vh_init_trento(h->context(), &ic, norms), h->context());
    h->adoptDeviceState();
    return {norms[0], norms[1]};
  }
};

// ICGubser (icModel 4)
class ICGubser {
 public:
  void setIC(Hydro* h) {
    check(vh_init_gubser(h->context()), h->context());
    h->adoptDeviceState();
  }
};

// IC (icModel 2) over the table of s95p::loadSongIC: "NX NY" then NX*NY
// lines "x y value" (src/s95p.cpp:43-66); glauberVar 1 reads entropy
class IC {
  std::vector<double> x_, y_, val_;
  int nx_ = 0, ny_ = 0;
  double factor_;
  int glauberVar_;

 public:
  IC(const char* icInputFile, double s0ScaleFactor, int glauberVar = 1)
      : factor_(s0ScaleFactor), glauberVar_(glauberVar) {
    std::ifstream fin(icInputFile);
    if (!fin) throw Error(VH_ERR_ARG, std::string("cannot open ") + icInputFile);
    fin >> nx_ >> ny_;
    if (nx_ < 2 || ny_ < 2) throw Error(VH_ERR_ARG, std::string("bad table size in ") + icInputFile);
    x_.assign(nx_, 0.);
    y_.assign(ny_, 0.);
    val_.assign((size_t)nx_ * ny_, 0.);
    for (int ix = 0; ix < nx_; ix++)
      for (int iy = 0; iy < ny_; iy++) fin >> x_[ix] >> y_[iy] >> val_[(size_t)ix * ny_ + iy];
  }
  const std::vector<double>& x() const { return x_; }
  const std::vector<double>& y() const { return y_; }
  const std::vector<double>& val() const { return val_; }
  void setIC(Hydro* h) {
    vh_table_ic ic{nx_, ny_, x_.data(), y_.data(), val_.data(), factor_, glauberVar_};
    check(vh_init_table(h->context(), &ic), h->context());
    h->adoptDeviceState();
  }
};

// IcPartUrqmd (icModel 3): "tau x y eta mt px py rap id charge" lines, a
// line that does not parse ending an event that holds particles
// (src/icPartUrqmd.cpp:79-103)
class IcPartUrqmd {
  std::vector<double> p_;
  std::vector<int> id_, charge_, npart_;
  double Rgt_, Rgz_;

 public:
  IcPartUrqmd(Fluid*, const char* filename, double Rgt, double Rgz, double /*tau0: the Hydro's*/)
      : Rgt_(Rgt), Rgz_(Rgz) {
    std::ifstream fin(filename);
    if (!fin.good()) throw Error(VH_ERR_ARG, std::string("I/O error with ") + filename);
    std::string line;
    int np = 0;
    while (!fin.eof()) {  // as IcGlissando's reader: see there for the last line
      std::getline(fin, line);
      std::istringstream in(line);
      double v[8];
      int id, ch;
      if (in >> v[0] >> v[1] >> v[2] >> v[3] >> v[4] >> v[5] >> v[6] >> v[7] >> id >> ch) {
        p_.insert(p_.end(), v, v + 8);
        id_.push_back(id);
        charge_.push_back(ch);
        if (++np > 9999) throw Error(VH_ERR_ARG, "IcPartUrqmd: more particles in an event than NP");
      } else if (np > 0) {
        npart_.push_back(np);
        np = 0;
      }
    }
    if (npart_.empty()) throw Error(VH_ERR_ARG, std::string("no particle events in ") + filename);
  }
  int nevents() const { return (int)npart_.size(); }
  const std::vector<int>& npart() const { return npart_; }
  void setIC(Hydro* h) {
    vh_urqmd_ic ic{p_.data(), id_.data(), charge_.data(), npart_.data(), nevents(), Rgt_, Rgz_};
    check(vh_init_urqmd(h->context(), &ic), h->context());
    h->adoptDeviceState();
  }
};

// ------------------------------------------------------------- parameters
// The reference driver's parameters with their defaults (src/main.cpp:70-81)
// and its params-file reader (src/main.cpp:83-156): "name value" lines;
// lines starting with '!' are comments echoed as "CCC", unknown names are
// echoed as "UUU"; the grid must have min < max on every axis.
struct Params {
  int nx = 100, ny = 100, nz = 100, eosType = 1, etaSparam = 0, zetaSparam = 0,
      eosTypeHadron = 0;
  bool freezeoutOnly = false, freezeoutExtend = false, vorticityOn = false;
  double xmin = -5.0, xmax = 5.0, ymin = -5.0, ymax = 5.0, etamin = -5.0, etamax = 5.0,
         tau0 = 1.0, tauMax = 20.0, tauResize = 4.0, dtau = 0.05, etaS = 0.08, zetaS = 0.0,
         eCrit = 0.5, etaSEpsilonMin = 5., al = 0., ah = 0., aRho = 0., T0 = 0.15,
         etaSMin = 0.08, etaSShiftMuB = 0., etaSScaleMuB = 0., zetaSPeakEpsilon = 5.,
         zetaSScaleBeta = 0.103, zetaSSigmaMinus = 0.1, zetaSSigmaPlus = 0.1, epsilon0 = 0.,
         Rgt = 1.0, Rgz = 1.0, impactPar = 0., s0ScaleFactor = 0.;
  std::string collSystem, outputDir = "data", isInputFile, vtk_values;
  int icModel = 1, glauberVariable = 1, smoothingType = 0;
  // not a reference parameter: an EoS1f table for the hydro EoS (the
  // reference selects compiled-in EoS classes with eosType instead)
  std::string eos1fFile;

  void read(const char* parFile, std::ostream& log) {
    std::ifstream fin(parFile);
    if (!fin.is_open()) throw Error(VH_ERR_ARG, std::string("cannot open parameters file ") + parFile);
    auto I = [](int& v) { return [&v](const std::string& s) { v = atoi(s.c_str()); }; };
    auto D = [](double& v) { return [&v](const std::string& s) { v = atof(s.c_str()); }; };
    auto B = [](bool& v) { return [&v](const std::string& s) { v = atoi(s.c_str()); }; };
    auto S = [](std::string& v) { return [&v](const std::string& s) { v = s; }; };
    std::map<std::string, std::function<void(const std::string&)>> h = {
        {"eosType", I(eosType)}, {"eosTypeHadron", I(eosTypeHadron)}, {"nx", I(nx)},
        {"ny", I(ny)}, {"nz", I(nz)}, {"icModel", I(icModel)},
        {"glauberVar", I(glauberVariable)}, {"xmin", D(xmin)}, {"xmax", D(xmax)},
        {"ymin", D(ymin)}, {"ymax", D(ymax)}, {"etamin", D(etamin)}, {"etamax", D(etamax)},
        {"tau0", D(tau0)}, {"tauMax", D(tauMax)}, {"tauGridResize", D(tauResize)},
        {"dtau", D(dtau)}, {"e_crit", D(eCrit)}, {"etaS", D(etaS)}, {"zetaS", D(zetaS)},
        {"zetaSparam", I(zetaSparam)}, {"zetaSScaleBeta", D(zetaSScaleBeta)},
        {"zetaSPeakEpsilon", D(zetaSPeakEpsilon)}, {"zetaSSigmaMinus", D(zetaSSigmaMinus)},
        {"zetaSSigmaPlus", D(zetaSSigmaPlus)}, {"epsilon0", D(epsilon0)}, {"Rg", D(Rgt)},
        {"Rgz", D(Rgz)}, {"impactPar", D(impactPar)}, {"s0ScaleFactor", D(s0ScaleFactor)},
        {"VTK_output_values", S(vtk_values)}, {"etaSparam", I(etaSparam)}, {"aRho", D(aRho)},
        {"ah", D(ah)}, {"al", D(al)}, {"T0", D(T0)}, {"etaSEpsilonMin", D(etaSEpsilonMin)},
        {"etaSMin", D(etaSMin)}, {"etaSShiftMuB", D(etaSShiftMuB)},
        {"etaSScaleMuB", D(etaSScaleMuB)}, {"freezeoutOnly", B(freezeoutOnly)},
        {"freezeoutExtend", B(freezeoutExtend)}, {"vorticity", B(vorticityOn)},
        {"smoothingType", I(smoothingType)}, {"eos1fFile", S(eos1fFile)},
    };
    // as in the reference, a line's name and value go through fixed
    // buffers that keep their previous contents when a line has fewer words
    std::string name, value;
    while (fin.good()) {
      std::string line;
      std::getline(fin, line);
      std::istringstream sline(line);
      std::string a, b;
      if (sline >> a) name = a;
      if (sline >> b) value = b;
      auto it = h.find(name);
      if (it != h.end())
        it->second(value);
      else if (!name.empty() && name[0] == '!')
        log << "CCC " << line << "\n";
      else
        log << "UUU " << line << "\n";
    }
    if (!(xmin < xmax)) throw Error(VH_ERR_ARG, "The hydrodynamic grid is not set up correctly: xmin >= xmax");
    if (!(ymin < ymax)) throw Error(VH_ERR_ARG, "The hydrodynamic grid is not set up correctly: ymin >= ymax");
    if (!(etamin < etamax)) throw Error(VH_ERR_ARG, "The hydrodynamic grid is not set up correctly: etamin >= etamax");
  }
};

}  // namespace vhb
