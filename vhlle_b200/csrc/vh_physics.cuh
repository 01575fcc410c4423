// vh_physics.cuh -- per-cell / per-face FP64 physics of the vHLLE step,
// as device functions.
//
// Every function keeps the operation order of the reference function cited
// in its comment, and the library is compiled with -fmad=false, so that
// IEEE-754 double arithmetic gives the reference's results bit for bit
// (division and square root are correctly rounded on both sides).
#pragma once

#include <cstdint>

#include "vh_crmath.cuh"

namespace vh {

enum { T_ = 0, X_ = 1, Y_ = 2, Z_ = 3, NB_ = 4, NQ_ = 5, NS_ = 6 };

// error bits (the reference exits on these conditions)
enum : unsigned {
  ERR_E_HUGE = 1u,       // e > 1e10 in hlle_flux, src/hdo.cpp:118-130
  ERR_FLUX_NAN = 2u,     // src/hdo.cpp:285-298
  ERR_SOURCE_NAN = 4u,   // src/hdo.cpp:345-351
  ERR_NSQUANT_NAN = 8u,  // src/hdo.cpp:643-651
  ERR_SURFACE = 16u,     // Cornelius would stop the reference (src/cornelius.cpp:1217,1534)
};

// How a table axis is searched: a binary search as the reference does, or
// an index guess from the axis' log or linear spacing followed by a walk to
// the same bracket (GRID_LOG / GRID_LIN need a strictly increasing axis).
enum : int { GRID_BSEARCH = 0, GRID_LOG = 1, GRID_LIN = 2 };

// One EoSChiral sub-table (EoSaux): uniform grids, p/T/mub/mus[in*ne + ie]
struct ChiralAux {
  int ne, nn;
  double emin, emax, nmin, nmax;
  const double *__restrict__ p, *__restrict__ T, *__restrict__ mub, *__restrict__ mus;
};

// EoSHadron's tables and constants (kind 4, the freeze-out EoS):
// p/T/mub/muq/mus and status at [inq + nnq*inb + nnq*nnb*ie]
struct HadronTab {
  int ne, nnb, nnq;
  double e0, n0, logemin, logemax, lognmax;
  double nb_abs_min, nq_abs_min, e_min;  // the constructor's derived constants
  const double *__restrict__ p, *__restrict__ T, *__restrict__ mub, *__restrict__ muq,
      *__restrict__ mus;
  const int* __restrict__ status;
};

// EoSSmash's tables and grids (kind 5, a freeze-out EoS)
struct SmashTab {
  int ne, nnb, nnq;
  double emin, emax, nbmin, nbmax, nqmin, nqmax;
  const double *__restrict__ p, *__restrict__ T, *__restrict__ mub, *__restrict__ muq,
      *__restrict__ mus;
};

// one of EoSAZH's six tables (EoSAZHaux, src/eoAZH.cpp:15-56): ne x nn
// values at [ie * nn + in] on the uniform grids emin + ie de, nmin + in dn
struct AzhTab {
  int ne, nn;
  double emin, nmin, de, dn;
  const double* __restrict__ v;
};

struct EosDev {
  int kind;          // 0 conformal gas, 1 EoS1f (e, nb) table, 2 EoSChiral
  double conf_cnst;  // e = cnst T^4 for kind 0
  int ne, nn;
  const double* __restrict__ egrid;
  const double* __restrict__ ngrid;
  const double* __restrict__ p;  // [ie + ne*inb]
  const double* __restrict__ T;
  const double* __restrict__ mub;
  int emode, nmode;    // GRID_* per axis
  float e0, einv;      // guess: (f(x) - e0) * einv, f = log2 or identity
  float n0, ninv;
  // RN(1 / (g[k+1] - g[k])) per interval of each axis, or null: the
  // interpolation weights then take crm::mk_div instead of a divide
  const double* __restrict__ erinv;
  const double* __restrict__ nrinv;
  // con2prim policy (not part of the EoS proper, but passed everywhere with
  // it): stop when |dv| < tol (the reference's 0.00001 by default); vguess,
  // when set, holds a start point in (0, 1) per cell for the root find; stats,
  // when set, counts calls [0] and iterations [1].
  double tol;
  const float* __restrict__ vguess;
  unsigned long long* stats;
  // the Newton slope of the root find: 0 the reference's constant
  // dp/de = 1/3; 1 the EoS's own local dp/de and dp/dnb (the step kernels
  // take it through the EK_*_SL instantiations)
  int slope;
  ChiralAux ch[2];  // kind 2: chiralsmall, chiraleos
  // kind 3 (EoS3f): muQ and muS tables beside p, T, muB (the 4-D layout
  // [ie + ne*ib + ne*nn*iq + ne*nn*nn*is]); iq0 and uq0 are the n-grid
  // bracket and weight of a zero charge, the nq and ns of every lookup
  const double* __restrict__ muq;
  const double* __restrict__ mus;
  int iq0;
  double uq0;
  HadronTab h;  // kind 4
  SmashTab sm;  // kind 5
  AzhTab az[6];  // kind 6: p1, p2, T1, T2, mu1, mu2
};

__device__ __forceinline__ float c2p_guess(const EosDev& E, long long i) {
  return E.vguess ? E.vguess[i] : -1.f;
}

struct TrDev {
  double etaS0, zetaS0, ah, al, aRho, T0, etaSMin, etaSEpsilonMin,
      etaSShiftMuB, etaSScaleMuB, zetaSPeakEpsilon, zetaSScaleBeta,
      zetaSSigmaMinus, zetaSSigmaPlus;
  int etaSparam, zetaSparam;
  double zetaSPeakT, zetaSWidthT;  // zetaSparam 5
};

struct Prim {
  double e, p, nb, nq, ns, vx, vy, vz;
};

__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

// index44, src/cll.cpp:22-31
__host__ __device__ __forceinline__ int index44(int i, int j) {
  return (j < i) ? (i * (i + 1)) / 2 + j : (j * (j + 1)) / 2 + i;
}

// minmod, src/cll.cpp:12-19
__device__ __forceinline__ double minmod(double a, double b) {
  if (a * b <= 0.) return 0.;
  return (fabs(a) > fabs(b)) ? b : a;
}

// ---------------------------------------------- zero-safe FP64 division
// On B200 an FP64 division (or square root) of zero leaves the operation's
// fast path and costs about three times a regular one, and one such lane
// holds up its whole warp.  This step divides zeros all the time (nb = 0 in
// every EoS lookup of a baryon-free run, vanishing velocity components, zero
// tensor entries and coefficients).  The helpers below return exactly the
// IEEE-754 result, but never hand the hardware a zero operand: the operand
// is swapped for 1.0 by a PTX select, which the compiler cannot see through
// (a plain C select would be folded back into the original division), and
// the result for a zero operand is formed from the signs.
__device__ __forceinline__ double one_if(bool z, double y) {
  double r;
  asm("{\n\t.reg .pred p;\n\tsetp.ne.s32 p, %2, 0;\n\tselp.f64 %0, 0d3FF0000000000000, %1, p;\n\t}"
      : "=d"(r)
      : "d"(y), "r"((int)z));
  return r;
}

// y / b
__device__ __forceinline__ double ddiv(double y, double b) {
  const bool z = (y == 0.);
  const double q = one_if(z, y) / b;
  if (!z) return q;
  return (b == 0. || b != b) ? q * y : (signbit(b) ? -y : y);
}

// y / b for a divisor known to be positive (finite or +inf)
__device__ __forceinline__ double ddivp(double y, double b) {
  const bool z = (y == 0.);
  const double q = one_if(z, y) / b;
  return z ? y : q;
}

// n[j] <- ddivp(n[j], b) (ddiv with GENERAL) for j < K, r = RN(1/b):
// through crm::mk_div when every numerator and b are in its range
// (bit-identical to either, b being positive there; no divide), else with
// the divide.
template <int K, bool GENERAL = false>
__device__ __forceinline__ void div_batch(double* n, double b, double r, bool bfast) {
  bool ok = bfast;
#pragma unroll
  for (int j = 0; j < K; j++) ok = ok && crm::mk_num_ok(n[j]);
  if (ok) {
#pragma unroll
    for (int j = 0; j < K; j++) n[j] = crm::mk_div(n[j], b, r);
  } else {
#pragma unroll
    for (int j = 0; j < K; j++) n[j] = GENERAL ? ddiv(n[j], b) : ddivp(n[j], b);
  }
}

// the 7 components of Q / t (t > 0) into q, through div_batch
__device__ __forceinline__ void q_over(const double* qin, double t, double* q) {
#pragma unroll
  for (int k = 0; k < 7; k++) q[k] = qin[k];
  div_batch<7>(q, t, 1.0 / t, crm::mk_den_ok(t));
}

// sqrt(x) (sqrt(+-0) = +-0)
__device__ __forceinline__ double sqrtz(double x) {
  const bool z = (x == 0.);
  const double r = sqrt(one_if(z, x));
  return z ? x : r;
}

// ------------------------------------------------------------------ EoS
// EoS1f binary search over a sorted grid (getue / getun, src/eo1.cpp:63-98);
// returns k1 of the bracketing pair and k2.
__device__ __forceinline__ void bsearch_grid(const double* __restrict__ g, int n,
                                             double x, int& k1, int& k2) {
  k1 = 0;
  k2 = n - 1;
  while (k2 - k1 > 1) {
    const int k = (k1 + k2) / 2;
    if (x < __ldg(g + k))
      k2 = k;
    else
      k1 = k;
  }
}

// The bracket the binary search above returns, found from an index guess.
// (x - g0) / (g1 - g0) for the bracket [g0, g1] of an axis: with the
// interval's reciprocal r (computed on the host by the same subtraction and
// a divide; has_r false without a table) through crm::mk_div,
// bit-identical to the divide, when x - g0 is in its range; else divided.
__device__ __forceinline__ double interp_weight(double x, double g0, double g1, bool has_r,
                                                double r) {
  const double num = x - g0, den = g1 - g0;
  if (has_r && crm::mk_num_ok(num)) return crm::mk_div(num, den, r);
  return ddiv(num, den);
}

// The float guess of a GRID_LOG / GRID_LIN axis position, in [0, n-2].
__device__ __forceinline__ int axis_guess(int n, double x, int mode, float x0, float inv) {
  if (x != x) return n - 2;
  const float fx = (float)x;
  const float t = (mode == GRID_LOG ? __log2f(fx) - x0 : fx - x0) * inv;
  return !(t > 0.f) ? 0 : (t >= (float)(n - 2) ? n - 2 : (int)t);
}

// k is bsearch_grid's bracket of x when (k == 0 or g[k] <= x) and
// (k == n-2 or x < g[k+1]) (NaN: k == n-2).
__device__ __forceinline__ bool is_bracket(int k, int n, double x, double gk, double gk1) {
  return (k == 0 || !(x < gk)) && (k == n - 2 || x < gk1);
}

// EoS1f::eos, src/eo1.cpp:100-123.  Both axes' brackets are guessed
// without loads (or searched, for an axis without a guess), and the bracket
// ends, the interval reciprocals and the four table corners are loaded
// together for the guess; a wrong guess (a step or two off, rare) walks to
// the bracket that the binary search finds and loads again.
// With WANT_D also the interpolant's partial derivatives dp/de and dp/dnb
// in the bracket (0 where p is clamped at 0): the Newton slope of the
// table-slope root find.
template <bool WANT_T, bool WANT_D = false>
__device__ __forceinline__ void eos1f(const EosDev& E, double e, double nb,
                                      double& T, double& mub, double& p, double* dpde = nullptr,
                                      double* dpdn = nullptr) {
  const int ne = E.ne, nn = E.nn;
  int ke, kn, k2;
  if (E.emode == GRID_BSEARCH || ne <= 2)
    bsearch_grid(E.egrid, ne, e, ke, k2);
  else
    ke = axis_guess(ne, e, E.emode, E.e0, E.einv);
  if (nn <= 2)
    kn = 0;
  else if (E.nmode == GRID_BSEARCH)
    bsearch_grid(E.ngrid, nn, nb, kn, k2);
  else
    kn = axis_guess(nn, nb, E.nmode, E.n0, E.ninv);
  double ge0 = __ldg(E.egrid + ke), ge1 = __ldg(E.egrid + ke + 1);
  double gn0 = __ldg(E.ngrid + kn), gn1 = __ldg(E.ngrid + kn + 1);
  double re = E.erinv ? __ldg(E.erinv + ke) : 0., rn = E.nrinv ? __ldg(E.nrinv + kn) : 0.;
  if (!is_bracket(ke, ne, e, ge0, ge1) || !is_bracket(kn, nn, nb, gn0, gn1)) {
    while (ke > 0 && e < __ldg(E.egrid + ke)) ke--;
    while (ke < ne - 2 && !(e < __ldg(E.egrid + ke + 1))) ke++;
    while (kn > 0 && nb < __ldg(E.ngrid + kn)) kn--;
    while (kn < nn - 2 && !(nb < __ldg(E.ngrid + kn + 1))) kn++;
    ge0 = __ldg(E.egrid + ke);
    ge1 = __ldg(E.egrid + ke + 1);
    gn0 = __ldg(E.ngrid + kn);
    gn1 = __ldg(E.ngrid + kn + 1);
    re = E.erinv ? __ldg(E.erinv + ke) : 0.;
    rn = E.nrinv ? __ldg(E.nrinv + kn) : 0.;
  }
  const int b00 = ke + ne * kn, b01 = ke + ne * (kn + 1);
  const double ue = interp_weight(e, ge0, ge1, E.erinv != nullptr, re);
  const double un = interp_weight(nb, gn0, gn1, E.nrinv != nullptr, rn);
  const double we0 = 1. - ue, we1 = ue;
  const double wn0 = 1. - un, wn1 = un;
  const double p00 = __ldg(E.p + b00), p01 = __ldg(E.p + b01);
  const double p10 = __ldg(E.p + b00 + 1), p11 = __ldg(E.p + b01 + 1);
  double sp = 0.;
  sp += we0 * wn0 * p00;
  sp += we0 * wn1 * p01;
  sp += we1 * wn0 * p10;
  sp += we1 * wn1 * p11;
  if (WANT_D) {
    const double se = wn0 * (p10 - p00) + wn1 * (p11 - p01);
    const double sn = we0 * (p01 - p00) + we1 * (p11 - p10);
    *dpde = sp < 0. ? 0. : (E.erinv ? se * re : ddiv(se, ge1 - ge0));
    *dpdn = sp < 0. ? 0. : (E.nrinv ? sn * rn : ddiv(sn, gn1 - gn0));
  }
  if (sp < 0.) sp = 0.;
  p = sp;
  if (WANT_T) {
    double sT = 0., sm = 0.;
    sT += we0 * wn0 * __ldg(E.T + b00);
    sT += we0 * wn1 * __ldg(E.T + b01);
    sT += we1 * wn0 * __ldg(E.T + b00 + 1);
    sT += we1 * wn1 * __ldg(E.T + b01 + 1);
    sm += we0 * wn0 * __ldg(E.mub + b00);
    sm += we0 * wn1 * __ldg(E.mub + b01);
    sm += we1 * wn0 * __ldg(E.mub + b00 + 1);
    sm += we1 * wn1 * __ldg(E.mub + b01 + 1);
    T = sT;
    mub = sm;
  }
}

// EoSaux::get / EoSaux::p, src/eoChiral.cpp:99-151: the bracket is the
// truncated (x - min) / step, clamped; the weights are (x - min - i step) /
// step.  (int) of a double saturates here and gives INT_MIN on the host
// for a large negative quotient alike; the region tests of eos_chiral keep
// positive quotients below the table size.
// EoSCMFe's constants (src/eoCMFe.h:10-11, src/eoCMFe.cpp:34-37)
#define VH_CMFE_EPS0 (146.51751415742 * 0.87326281)
#define VH_CMFE_N0 (0.15891 * 0.87272727)

// CMFE: EoSCMFeaux::get / ::p (src/eoCMFe.cpp:121-189), the same lookup
// with e below EPS_CUTOFF = 2e-2 giving zeros and a NaN pressure (a NaN
// table entry) replaced: zeros inside the tables' region, the conformal
// fallback outside it.
template <bool WANT_T, bool WANT_D = false, bool CMFE = false>
__device__ __forceinline__ void chiral_aux(const ChiralAux& A, double e, double nb, double& p,
                                           double& T, double& mub, double& mus,
                                           double* dpde = nullptr, double* dpdn = nullptr) {
  if (CMFE ? e < 2e-2 : e < 0.) {
    T = mub = mus = p = 0.;
    if (WANT_D) *dpde = *dpdn = 0.;
    return;
  }
  const double de = (A.emax - A.emin) / (A.ne - 1);
  const double dn = (A.nmax - A.nmin) / (A.nn - 1);
  int ie = (int)((e - A.emin) / de);
  int in = (int)((nb - A.nmin) / dn);
  if (ie < 0) ie = 0;
  if (in < 0) in = 0;
  if (ie > A.ne - 2) ie = A.ne - 2;
  if (in > A.nn - 2) in = A.nn - 2;
  const double em = e - A.emin - ie * de;
  const double nm = nb - A.nmin - in * dn;
  const double we0 = 1. - em / de, we1 = em / de;
  const double wn0 = 1. - nm / dn, wn1 = nm / dn;
  const int b00 = in * A.ne + ie, b01 = b00 + A.ne;  // [ie][in], [ie][in + 1]
  const double p00 = __ldg(A.p + b00), p01 = __ldg(A.p + b01);
  const double p10 = __ldg(A.p + b00 + 1), p11 = __ldg(A.p + b01 + 1);
  double sp = 0.;
  sp += we0 * wn0 * p00;
  sp += we0 * wn1 * p01;
  sp += we1 * wn0 * p10;
  sp += we1 * wn1 * p11;
  if (WANT_D) {
    *dpde = sp < 0. ? 0. : (wn0 * (p10 - p00) + wn1 * (p11 - p01)) / de;
    *dpdn = sp < 0. ? 0. : (we0 * (p01 - p00) + we1 * (p11 - p10)) / dn;
  }
  if (WANT_T) {
    double sT = 0., sb = 0., ss = 0.;
    sT += we0 * wn0 * __ldg(A.T + b00);
    sb += we0 * wn0 * __ldg(A.mub + b00);
    ss += we0 * wn0 * __ldg(A.mus + b00);
    sT += we0 * wn1 * __ldg(A.T + b01);
    sb += we0 * wn1 * __ldg(A.mub + b01);
    ss += we0 * wn1 * __ldg(A.mus + b01);
    sT += we1 * wn0 * __ldg(A.T + b00 + 1);
    sb += we1 * wn0 * __ldg(A.mub + b00 + 1);
    ss += we1 * wn0 * __ldg(A.mus + b00 + 1);
    sT += we1 * wn1 * __ldg(A.T + b01 + 1);
    sb += we1 * wn1 * __ldg(A.mub + b01 + 1);
    ss += we1 * wn1 * __ldg(A.mus + b01 + 1);
    T = sT;
    mub = sb;
    mus = ss;
  }
  if (CMFE && isnan(sp)) {
    if (e > 0.8 * VH_CMFE_EPS0 || nb > 40. * VH_CMFE_N0) {
      sp = 0.2964 * e;
      if (WANT_T) {
        T = 0.15120476935 * crm::root4_cr(e);
        mub = mus = 0.0;
      }
    } else {
      sp = 0.;
      if (WANT_T) T = mub = mus = 0.;
    }
  }
  if (sp < 0.0) sp = 0.0;
  p = sp;
}

// EoSChiral::eos / EoSChiral::p, src/eoChiral.cpp:159-178 (muq = 0); the
// 1/4 power of the region above the tables is the correctly rounded one
template <bool WANT_T, bool WANT_D = false>
__device__ __forceinline__ void eos_chiral(const EosDev& E, double e, double nb, double& T,
                                           double& mub, double& mus, double& p,
                                           double* dpde = nullptr, double* dpdn = nullptr) {
  if (e < 1.46 && nb < 0.3) {
    chiral_aux<WANT_T, WANT_D>(E.ch[0], e, nb, p, T, mub, mus, dpde, dpdn);
  } else if (e < 146. && nb < 6.) {
    chiral_aux<WANT_T, WANT_D>(E.ch[1], e, nb, p, T, mub, mus, dpde, dpdn);
  } else {
    p = 0.2964 * e;
    if (WANT_D) {
      *dpde = 0.2964;
      *dpdn = 0.;
    }
    if (WANT_T) {
      T = 0.15120476935 * crm::root4_cr(e);
      mub = mus = 0.0;
    }
  }
}

// EoSCMFe::eos / ::p, src/eoCMFe.cpp:204-226 (muq = 0): the small table
// below 15 EPS_0 / 1000 and 5 N_0, the big one below 0.8 EPS_0 and 40 N_0,
// the conformal fallback (correctly rounded 1/4 power) above
template <bool WANT_T>
__device__ __forceinline__ void eos_cmfe(const EosDev& E, double e, double nb, double& T,
                                         double& mub, double& mus, double& p) {
  if (e < 15 * VH_CMFE_EPS0 / 1000.0 && nb < 5 * VH_CMFE_N0) {
    chiral_aux<WANT_T, false, true>(E.ch[0], e, nb, p, T, mub, mus);
  } else if (e < 0.8 * VH_CMFE_EPS0 && nb < 40. * VH_CMFE_N0) {
    chiral_aux<WANT_T, false, true>(E.ch[1], e, nb, p, T, mub, mus);
  } else {
    p = 0.2964 * e;
    if (WANT_T) {
      T = 0.15120476935 * crm::root4_cr(e);
      mub = mus = 0.0;
    }
  }
}

// EK selects the EoS kinds compiled in: EK_ANY (every kind, chosen at run
// time), EK_TABLE (kinds 0 and 1) or EK_CHIRAL (kind 2).  The step's
// con2prim kernels are instantiated per class: compiled into every
// con2prim iteration next to the table lookup, the chiral lookup made those
// kernels spill more (face kernels 25 % slower on the table kind).
// EK_TABLE_SL / EK_CHIRAL_SL: the same classes with the table-slope root
// find (EosDev::slope = 1); EK_TABLE3: EoS3f (kind 3); EK_HADRON:
// EoSHadron (kind 4, the surface's); EK_SMASH: EoSSmash (kind 5, the
// surface's); EK_AZH: EoSAZH (kind 6); EK_CMFE: EoSCMFe (kind 7).
enum {
  EK_ANY = -1, EK_TABLE = 1, EK_CHIRAL = 2, EK_TABLE_SL = 3, EK_CHIRAL_SL = 4, EK_TABLE3 = 5,
  EK_HADRON = 6, EK_SMASH = 7, EK_AZH = 8, EK_CMFE = 9
};
__host__ __device__ constexpr bool ek_chiral(int ek) { return ek == EK_CHIRAL || ek == EK_CHIRAL_SL; }
__host__ __device__ constexpr bool ek_slope(int ek) { return ek == EK_TABLE_SL || ek == EK_CHIRAL_SL; }

// p and its partial derivatives (the table-slope root find)
template <int EK = EK_ANY>
__device__ __forceinline__ double eos_p_d(const EosDev& E, double e, double nb, double& dpde,
                                          double& dpdn) {
  double T, mub, mus, p;
  if (ek_chiral(EK) || (EK == EK_ANY && E.kind == 2)) {
    eos_chiral<false, true>(E, e, nb, T, mub, mus, p, &dpde, &dpdn);
    return p;
  }
  if (E.kind == 0) {
    dpde = 1. / 3.;
    dpdn = 0.;
    return ddivp(e, 3.);
  }
  eos1f<false, true>(E, e, nb, T, mub, p, &dpde, &dpdn);
  return p;
}

// EoS3f::eos, src/eo3.cpp:132-175, at nq = ns = 0 (their bracket iq0 and
// weight uq0 are fixed): the binary searches of getue / getun (the e index
// clamped from above only; the weights from the unclamped bracket), then
// the 16 corners in the reference's order with the weight product
// ((w_e w_nb) w_nq) w_ns.  For e < 0 the reference zeroes its outputs and
// interpolates anyway (no return), which is what this does.
template <bool WANT_T>
__device__ __forceinline__ void eos3f(const EosDev& E, double e, double nb, double& T,
                                      double& mub, double& muq, double& mus, double& p) {
  const int ne = E.ne, nn = E.nn;
  int k1, k2;
  bsearch_grid(E.egrid, ne, e, k1, k2);
  const int ixe = k1 > ne - 2 ? ne - 2 : k1;
  const double ue = (e - __ldg(E.egrid + k1)) / (__ldg(E.egrid + k2) - __ldg(E.egrid + k1));
  bsearch_grid(E.ngrid, nn, nb, k1, k2);
  int ixb = k1 > nn - 2 ? nn - 2 : k1;
  if (ixb < 0) ixb = 0;
  const double ub = (nb - __ldg(E.ngrid + k1)) / (__ldg(E.ngrid + k2) - __ldg(E.ngrid + k1));
  const double we[2] = {1. - ue, ue}, wb[2] = {1. - ub, ub};
  const double wq[2] = {1. - E.uq0, E.uq0};
  const long long sb = ne, sq = (long long)ne * nn, ss = (long long)ne * nn * nn;
  double sp = 0., sT = 0., smb = 0., smq = 0., sms = 0.;
#pragma unroll
  for (int je = 0; je < 2; je++)
#pragma unroll
    for (int jb = 0; jb < 2; jb++)
#pragma unroll
      for (int jq = 0; jq < 2; jq++)
#pragma unroll
        for (int js = 0; js < 2; js++) {
          const long long k = (ixe + je) + sb * (ixb + jb) + sq * (E.iq0 + jq) + ss * (E.iq0 + js);
          const double w = we[je] * wb[jb] * wq[jq] * wq[js];
          sp += w * __ldg(E.p + k);
          if (WANT_T) {
            sT += w * __ldg(E.T + k);
            smb += w * __ldg(E.mub + k);
            smq += w * __ldg(E.muq + k);
            sms += w * __ldg(E.mus + k);
          }
        }
  if (sp < 0.) sp = 0.;
  p = sp;
  if (WANT_T) {
    T = sT;
    mub = smb;
    muq = smq;
    mus = sms;
  }
}

// EoSHadron's position of a charge on its table (the inverse log mapping
// of src/eoHadron.cpp:97-112)
__device__ __forceinline__ double hadron_x(double n, double n0, double lognmax, double dxn,
                                           double n_abs_min) {
  if (n != 0.0) {
    const double zn = crm::log_cr(fabs(n) / n0);
    if (zn >= -lognmax + 2.0 * dxn) return n / fabs(n) * 0.5 * (zn + lognmax);
    return n / n_abs_min * dxn;
  }
  return 0.;
}

// EoSHadron::eos / ::p, src/eoHadron.cpp:81-208, at nq = 0; its logarithms
// correctly rounded (crm::log_cr), the C library's value bar the rare
// arguments where the library itself misrounds: the pressure feeds
// transformPV's root search at the freeze-out surface, whose iteration count
// follows the last bit
template <bool WANT_T>
__device__ __forceinline__ void eos_hadron(const HadronTab& H, double e, double nb, double& T,
                                           double& mub, double& muq, double& mus, double& p) {
  const int ne = H.ne, nnb = H.nnb, nnq = H.nnq;
  auto ix3 = [&](int ie, int inb, int inq) {
    return (long long)inq + (long long)nnq * inb + (long long)nnq * nnb * ie;
  };
  T = mub = muq = mus = p = 0.;
  if (e <= 0.) return;
  if (e < H.e_min) {
    p = e / H.e_min * __ldg(H.p + ix3(0, nnb / 2, nnq / 2));
    if (WANT_T) T = e / H.e_min * __ldg(H.T + ix3(0, nnb / 2, nnq / 2));
    return;
  }
  const double xe = crm::log_cr(e / H.e0);
  const double dxe = (H.logemax - H.logemin) / (ne - 1);
  const double dxnb = (2.0 * H.lognmax) / (nnb - 1);
  const double dxnq = (2.0 * H.lognmax) / (nnq - 1);
  const double xnb = hadron_x(nb, H.n0, H.lognmax, dxnb, H.nb_abs_min);
  const double xnq = 0.;  // nq = 0
  int ie = (int)((xe - H.logemin) / dxe);
  int inb = (int)((xnb + H.lognmax) / dxnb);
  int inq = (int)((xnq + H.lognmax) / dxnq);
  if (ie < 0) ie = 0;
  if (inb < 0) inb = 0;
  if (inq < 0) inq = 0;
  if (ie > ne - 2) ie = ne - 2;
  if (inb > nnb - 2) inb = nnb - 2;
  if (inq > nnq - 2) inq = nnq - 2;
  const double em = xe - H.logemin - ie * dxe;
  const double nbm = xnb + H.lognmax - inb * dxnb;
  const double nqm = xnq + H.lognmax - inq * dxnq;
  if (__ldg(H.status + ix3(ie, inb, inq)) == 1) return;
  const double we[2] = {1. - em / dxe, em / dxe};
  const double wnb[2] = {1. - nbm / dxnb, nbm / dxnb};
  const double wnq[2] = {1. - nqm / dxnq, nqm / dxnq};
  double sp = 0., sT = 0., sb = 0., sq = 0., ss = 0.;
#pragma unroll
  for (int je = 0; je < 2; je++)
#pragma unroll
    for (int jnb = 0; jnb < 2; jnb++)
#pragma unroll
      for (int jnq = 0; jnq < 2; jnq++) {
        const long long k = ix3(ie + je, inb + jnb, inq + jnq);
        sp += we[je] * wnb[jnb] * wnq[jnq] * __ldg(H.p + k);
        if (WANT_T) {
          sT += we[je] * wnb[jnb] * wnq[jnq] * __ldg(H.T + k);
          sb += we[je] * wnb[jnb] * wnq[jnq] * __ldg(H.mub + k);
          sq += we[je] * wnb[jnb] * wnq[jnq] * __ldg(H.muq + k);
          ss += we[je] * wnb[jnb] * wnq[jnq] * __ldg(H.mus + k);
        }
      }
  if (sp < 0.0) sp = 0.0;
  p = sp;
  if (WANT_T) {
    T = sT;
    mub = sb;
    muq = sq;
    mus = ss;
  }
}

// EoSSmash::eos / ::p, src/eoSmash.cpp:70-177, at nq = 0
template <bool WANT_T>
__device__ __forceinline__ void eos_smash(const SmashTab& H, double e, double nb, double& T,
                                          double& mub, double& muq, double& mus, double& p) {
  const int ne = H.ne, nnb = H.nnb, nnq = H.nnq;
  auto ix3 = [&](int ie, int inb, int inq) {
    return (long long)inq + (long long)nnq * inb + (long long)nnq * nnb * ie;
  };
  T = mub = muq = mus = p = 0.;
  if (e <= 0.) return;
  if (e < H.emin) {
    p = e / H.emin * __ldg(H.p + ix3(0, nnb / 2, nnq / 2));
    if (WANT_T) T = e / H.emin * __ldg(H.T + ix3(0, nnb / 2, nnq / 2));
    return;
  }
  const double nq = 0.;
  const double de = (H.emax - H.emin) / (ne - 1);
  const double dnb = (H.nbmax - H.nbmin) / (nnb - 1);
  const double dnq = (H.nqmax - H.nqmin) / (nnq - 1);
  int ie = (int)((e - H.emin) / de);
  int inb = (int)((nb - H.nbmin) / dnb);
  int inq = (int)((nq - H.nqmin) / dnq);
  if (ie < 0) ie = 0;
  if (inb < 0) inb = 0;
  if (inq < 0) inq = 0;
  if (ie > ne - 2) ie = ne - 2;
  if (inb > nnb - 2) inb = nnb - 2;
  if (inq > nnq - 2) inq = nnq - 2;
  const double em = e - H.emin - ie * de;
  const double nbm = nb - H.nbmin - inb * dnb;
  const double nqm = nq - H.nqmin - inq * dnq;
  const double we[2] = {1. - em / de, em / de};
  const double wnb[2] = {1. - nbm / dnb, nbm / dnb};
  const double wnq[2] = {1. - nqm / dnq, nqm / dnq};
  double sp = 0., sT = 0., sb = 0., sq = 0., ss = 0.;
#pragma unroll
  for (int je = 0; je < 2; je++)
#pragma unroll
    for (int jnb = 0; jnb < 2; jnb++)
#pragma unroll
      for (int jnq = 0; jnq < 2; jnq++) {
        const long long k = ix3(ie + je, inb + jnb, inq + jnq);
        sp += we[je] * wnb[jnb] * wnq[jnq] * __ldg(H.p + k);
        if (WANT_T) {
          sT += we[je] * wnb[jnb] * wnq[jnq] * __ldg(H.T + k);
          sb += we[je] * wnb[jnb] * wnq[jnq] * __ldg(H.mub + k);
          sq += we[je] * wnb[jnb] * wnq[jnq] * __ldg(H.muq + k);
          ss += we[je] * wnb[jnb] * wnq[jnq] * __ldg(H.mus + k);
        }
      }
  if (sp < 0.0) sp = 0.0;
  p = sp;
  if (WANT_T) {
    T = sT;
    mub = sb;
    muq = sq;
    mus = ss;
  }
}

// EoSAZHaux::get, src/eoAZH.cpp:58-83: bilinear in the cell of (e, nb),
// the cell clamped to the table (outside it the edge cell extrapolates)
__device__ __forceinline__ double azh_get(const AzhTab& t, double e, double nb) {
  if (e <= 0.) return 0.0;
  int ie = (int)((e - t.emin) / t.de);
  int in = (int)((nb - t.nmin) / t.dn);
  if (ie < 0) ie = 0;
  if (in < 0) in = 0;
  if (ie > t.ne - 2) ie = t.ne - 2;
  if (in > t.nn - 2) in = t.nn - 2;
  const double em = (e - t.emin - ie * t.de) / t.de;
  const double nm = (nb - t.nmin - in * t.dn) / t.dn;
  const double we[2] = {1. - em, em};
  const double wn[2] = {1. - nm, nm};
  double value = 0.0;
#pragma unroll
  for (int je = 0; je < 2; je++)
#pragma unroll
    for (int jn = 0; jn < 2; jn++)
      value += we[je] * wn[jn] * __ldg(t.v + (long long)(ie + je) * t.nn + (in + jn));
  return value;
}

// EoSAZHaux::getLow, src/eoAZH.cpp:85-102: below the table's e range, the
// first row linear in nb, scaled by e / emin.  (The reference exits when
// (nb - nmin) / dn > 10000; here the clamped first-row cell extrapolates.)
__device__ __forceinline__ double azh_low(const AzhTab& t, double e, double nb) {
  if (e <= 0.) return 0.0;
  int in = (int)((nb - t.nmin) / t.dn);
  if (in < 0) in = 0;
  if (in > t.nn - 2) in = t.nn - 2;
  const double nm = (nb - t.nmin - in * t.dn) / t.dn;
  const double wn[2] = {1. - nm, nm};
  const double value = wn[0] * __ldg(t.v + in) + wn[1] * __ldg(t.v + in + 1);
  return value * e / t.emin;
}

// EoSAZH::eos / ::p, src/eoAZH.cpp:123-150: the second table set above the
// first p table's e range, the first inside it, getLow below; p and T at
// |nb|, muB at nb; muQ = muS = 0
template <bool WANT_T>
__device__ __forceinline__ void eos_azh(const EosDev& E, double e, double nb, double& T,
                                        double& mub, double& p) {
  const AzhTab* a = E.az;
  const double anb = fabs(nb);
  T = mub = 0.;
  if (e > a[0].emin + a[0].de * (a[0].ne - 1)) {
    p = azh_get(a[1], e, anb);
    if (WANT_T) {
      T = azh_get(a[3], e, anb);
      mub = azh_get(a[5], e, nb);
    }
  } else if (e > a[0].emin) {
    p = azh_get(a[0], e, anb);
    if (WANT_T) {
      T = azh_get(a[2], e, anb);
      mub = azh_get(a[4], e, nb);
    }
  } else {
    p = azh_low(a[0], e, anb);
    if (WANT_T) {
      T = azh_low(a[2], e, anb);
      mub = azh_low(a[4], e, nb);
    }
  }
}

template <int EK = EK_ANY>
__device__ __forceinline__ double eos_p(const EosDev& E, double e, double nb) {
  double T, mub, mus, p;
  if (EK == EK_AZH || (EK == EK_ANY && E.kind == 6)) {
    eos_azh<false>(E, e, nb, T, mub, p);
    return p;
  }
  if (EK == EK_CMFE || (EK == EK_ANY && E.kind == 7)) {
    eos_cmfe<false>(E, e, nb, T, mub, mus, p);
    return p;
  }
  if (EK == EK_SMASH || (EK == EK_ANY && E.kind == 5)) {
    double muq;
    eos_smash<false>(E.sm, e, nb, T, mub, muq, mus, p);
    return p;
  }
  if (EK == EK_HADRON || (EK == EK_ANY && E.kind == 4)) {
    double muq;
    eos_hadron<false>(E.h, e, nb, T, mub, muq, mus, p);
    return p;
  }
  if (EK == EK_TABLE3 || (EK == EK_ANY && E.kind == 3)) {
    double muq;
    eos3f<false>(E, e, nb, T, mub, muq, mus, p);
    return p;
  }
  if (ek_chiral(EK) || (EK == EK_ANY && E.kind == 2)) {
    eos_chiral<false>(E, e, nb, T, mub, mus, p);
    return p;
  }
  if (E.kind == 0) return ddivp(e, 3.);
  eos1f<false>(E, e, nb, T, mub, p);
  return p;
}

// EoS::eos with muS (muQ is 0 for every kind here; muS only for kind 2)
template <int EK = EK_ANY>
__device__ __forceinline__ void eos_eval(const EosDev& E, double e, double nb, double& T,
                                         double& mub, double& mus, double& p) {
  mus = 0.;
  if (EK == EK_AZH || (EK == EK_ANY && E.kind == 6)) {
    eos_azh<true>(E, e, nb, T, mub, p);
  } else if (EK == EK_CMFE || (EK == EK_ANY && E.kind == 7)) {
    eos_cmfe<true>(E, e, nb, T, mub, mus, p);
  } else if (EK == EK_SMASH || (EK == EK_ANY && E.kind == 5)) {
    double muq;
    eos_smash<true>(E.sm, e, nb, T, mub, muq, mus, p);
  } else if (EK == EK_HADRON || (EK == EK_ANY && E.kind == 4)) {
    double muq;
    eos_hadron<true>(E.h, e, nb, T, mub, muq, mus, p);
  } else if (EK == EK_TABLE3 || (EK == EK_ANY && E.kind == 3)) {
    double muq;
    eos3f<true>(E, e, nb, T, mub, muq, mus, p);
  } else if (ek_chiral(EK) || (EK == EK_ANY && E.kind == 2)) {
    eos_chiral<true>(E, e, nb, T, mub, mus, p);
  } else if (E.kind == 0) {
    p = ddivp(e, 3.);
    T = e > 0. ? sqrt(sqrt(e / E.conf_cnst)) : 0.;
    mub = 0.;
  } else {
    eos1f<true>(E, e, nb, T, mub, p);
  }
}

template <int EK = EK_ANY>
__device__ __forceinline__ void eos_eval(const EosDev& E, double e, double nb,
                                         double& T, double& mub, double& p) {
  double mus;
  eos_eval<EK>(E, e, nb, T, mub, mus, p);
}

// EoS::eos with muQ, which only EoS3f has (0 for the other kinds)
template <int EK = EK_ANY>
__device__ __forceinline__ void eos_eval_q(const EosDev& E, double e, double nb, double& T,
                                           double& mub, double& muq, double& mus, double& p) {
  if (EK == EK_SMASH || (EK == EK_ANY && E.kind == 5)) {
    eos_smash<true>(E.sm, e, nb, T, mub, muq, mus, p);
    return;
  }
  if (EK == EK_HADRON || (EK == EK_ANY && E.kind == 4)) {
    eos_hadron<true>(E.h, e, nb, T, mub, muq, mus, p);
    return;
  }
  if (EK == EK_TABLE3 || (EK == EK_ANY && E.kind == 3)) {
    eos3f<true>(E, e, nb, T, mub, muq, mus, p);
    return;
  }
  muq = 0.;
  eos_eval<EK>(E, e, nb, T, mub, mus, p);
}

// EoS::s, src/eos.cpp:18-25
__device__ __forceinline__ double eos_s(const EosDev& E, double e, double nb,
                                        double nq, double ns) {
  double T, mub, mus, p, muq;
  eos_eval_q(E, e, nb, T, mub, muq, mus, p);
  if (T > 0.0) return ddivp(e + p - mub * nb - muq * nq - mus * ns, T);
  return 0.;
}

// ----------------------------------------------------------- transformPV
// src/rmn.cpp:28-139.  Q is the caller's copy and is rescaled in place when
// |M| > Q_t, exactly as the reference does.  With a start point g in (0, 1)
// (a learned guess) the iteration starts there instead of at 0.5 and the
// bracket is narrowed by the sign of f at g; the safeguarded Newton /
// bisection then runs as in the reference until |dv| < E.tol.
template <int EK = EK_ANY>
__device__ __forceinline__ void transform_pv(const EosDev& E, double Q[7], Prim& o,
                                             float g = -1.f) {
  const int MAXIT = 100;
  const double dpe = 1. / 3.;
  const double corrf = 0.9999;
  double v, vl = 0., vh = 1., dvold, dv, f, df;
  double M = sqrtz(Q[X_] * Q[X_] + Q[Y_] * Q[Y_] + Q[Z_] * Q[Z_]);
  if (Q[T_] <= 0.) {
    o.e = 0.; o.p = 0.;
    o.vx = o.vy = o.vz = 0.;
    o.nb = o.nq = o.ns = 0.;
    return;
  }
  if (M == 0.) {
    o.e = Q[T_];
    o.vx = 0.; o.vy = 0.; o.vz = 0.;
    o.nb = Q[NB_]; o.nq = Q[NQ_]; o.ns = Q[NS_];
    o.p = eos_p<EK>(E, o.e, o.nb);
    return;
  }
  if (M > Q[T_]) {
    Q[X_] *= corrf * Q[T_] / M;
    Q[Y_] *= corrf * Q[T_] / M;
    Q[Z_] *= corrf * Q[T_] / M;
    M = Q[T_] * corrf;
  }
  double e, p, nb, nq, ns;
  const bool guessed = g > 0.f && g < 1.f;
  v = guessed ? (double)g : 0.5 * (vl + vh);
  e = Q[T_] - M * v;
  if (e < 0.) e = 0.;
  {
    const double sq = sqrt(1 - v * v);
    nb = Q[NB_] * sq;
    nq = Q[NQ_] * sq;
    ns = Q[NS_] * sq;
  }
  // The table-slope variant (ek_slope) takes f' = (Q_t + p) - v (M dp/de +
  // dp/dnb Q_nb v / sqrt(1 - v^2)) with the EoS's own derivatives, so the
  // Newton steps converge quadratically inside a table cell, and stops when
  // f is exactly 0 (the reference's bracket test would send an exact root
  // into bisection).  Not the reference's iteration: for a tight tolerance
  // only, where the result does not depend on the path to the root.
  constexpr bool SL = ek_slope(EK);
  double dpde = 0., dpdn = 0.;
  auto slope = [&](double vv, double sq) {
    const double dn = sq > 0. ? dpdn * Q[NB_] * vv / sq : 0.;
    return (Q[T_] + p) - vv * (M * dpde + dn);
  };
  double sq0 = sqrt(1 - v * v);
  if (SL) {
    p = eos_p_d<EK>(E, e, nb, dpde, dpdn);
  } else {
    p = eos_p<EK>(E, e, nb);
  }
  f = (Q[T_] + p) * v - M;
  df = SL ? slope(v, sq0) : (Q[T_] + p) - M * v * dpe;
  if (guessed) {
    if (f > 0.)
      vh = v;
    else
      vl = v;
  }
  dvold = vh - vl;
  dv = dvold;
  int it = 0;
  const bool at_root = SL && f == 0.;  // a start point that is the root
  for (int i = 0; i < MAXIT && !at_root; i++) {
    it = i + 1;
    if ((f + df * (vh - v)) * (f + df * (vl - v)) >= 0. ||
        fabs(2. * f) > fabs(dvold * df)) {
      dvold = dv;
      dv = 0.5 * (vh - vl);
      v = vl + dv;
    } else {
      dvold = dv;
      dv = ddiv(f, df);
      v -= dv;
    }
    if (fabs(dv) < E.tol) break;
    e = Q[T_] - M * v;
    if (e < 0.) e = 0.;
    const double sq = sqrt(1 - v * v);
    nb = Q[NB_] * sq;
    nq = Q[NQ_] * sq;
    ns = Q[NS_] * sq;
    if (SL) {
      p = eos_p_d<EK>(E, e, nb, dpde, dpdn);
    } else {
      p = eos_p<EK>(E, e, nb);
    }
    f = (Q[T_] + p) * v - M;
    if (SL && f == 0.) break;
    df = SL ? slope(v, sq) : (Q[T_] + p) - M * v * dpe;
    if (f > 0.)
      vh = v;
    else
      vl = v;
  }
  if (E.stats) {
    atomicAdd(&E.stats[0], 1ull);
    atomicAdd(&E.stats[1], (unsigned long long)it);
  }
  {
    // v Q_i / M, i = x, y, z: one divide for RN(1/M) and crm::mk_div
    // (bit-identical) when all three are in its range
    const double nx = v * Q[X_], ny = v * Q[Y_], nz = v * Q[Z_];
    if (crm::mk_den_ok(M) && crm::mk_num_ok(nx) && crm::mk_num_ok(ny) && crm::mk_num_ok(nz)) {
      const double rM = 1.0 / M;
      o.vx = crm::mk_div(nx, M, rM);
      o.vy = crm::mk_div(ny, M, rM);
      o.vz = crm::mk_div(nz, M, rM);
    } else {
      o.vx = ddivp(nx, M);
      o.vy = ddivp(ny, M);
      o.vz = ddivp(nz, M);
    }
  }
  o.e = Q[T_] - M * v;
  o.p = eos_p<EK>(E, o.e, nb);  // the last iterate's nb, as the reference
  const double sq = sqrt(1 - o.vx * o.vx - o.vy * o.vy - o.vz * o.vz);
  o.nb = Q[NB_] * sq;
  o.nq = Q[NQ_] * sq;
  o.ns = Q[NS_] * sq;
}

// ------------------------------------------------- transport coefficients
// TransportCoeff::zetaS, src/trancoeff.cpp:19-66; cs2(e) = 1/3 (src/eos.h:37).
// exp and pow(x, 0.25) are correctly rounded (vh_crmath.cuh), the value the
// host library's half-ulp functions return in all but ~1e-3 of the calls.
__device__ __forceinline__ double tr_zetaS(const TrDev& t, double e, double T,
                                           double s, double P) {
  const double cs2e = 1. / 3.;
  const double T_p = 0.180, T_peak = 0.165, T_width = 0.010, B_norm = 0.24,
               B_width = 1.5, T_peak2 = 0.160, B_norm2 = 0.13, B1 = 0.01, B2 = 0.12;
  if (t.zetaSparam == 0) {
    // the denominator is >= 1, so a zero (or NaN) numerator is the result
    const double num = t.zetaS0 * (1. / 3. - cs2e);
    if (num == 0. || num != num) return num;
    return num / (crm::exp_cr((0.16 - T) / 0.001) + 1.);
  } else if (t.zetaSparam == 1) {
    if (T < 0.180)
      return 0.03 + (0.08 * crm::exp_cr(((T / T_p) - 1.) / (0.0025))) +
             (0.22 * crm::exp_cr(((T / T_p) - 1) / (0.022)));
    else if (T >= 0.180 && T < 0.200)
      return 27.55 * (T / T_p) - 13.45 - (13.77 * (T / T_p) * (T / T_p));
    else if (T >= 0.200)
      return 0.001 + (0.9 * crm::exp_cr(-((T / T_p) - 1.) / (0.0025))) +
             (0.25 * crm::exp_cr(-((T / T_p) - 1.) / (0.13)));
  } else if (t.zetaSparam == 2) {
    if (T > T_peak)
      return B_norm * ((B_width * B_width) /
                       ((((T / T_peak) - 1.) * ((T / T_peak) - 1.)) + (B_width * B_width)));
    else if (T <= T_peak)
      return B_norm * (crm::exp_cr(-((T - T_peak) / T_width) * ((T - T_peak) / T_width)));
  } else if (t.zetaSparam == 3) {
    if (T < T_peak2)
      return B_norm2 * crm::exp_cr(-((T - T_peak2) * (T - T_peak2) / (B1 * B1)));
    else if (T >= T_peak2)
      return B_norm2 * crm::exp_cr(-((T - T_peak2) * (T - T_peak2) / (B2 * B2)));
  } else if (t.zetaSparam == 4) {
    // abs(s) binds to int abs(int) in the reference: |s| < 1 reads as 0
    if (!(fabs(s) >= 1.0) || T < 1e-1) return 0;
    const double d = t.zetaSScaleBeta * (crm::root4_cr(e) - crm::root4_cr(t.zetaSPeakEpsilon));
    const double sig = e < t.zetaSPeakEpsilon ? t.zetaSSigmaMinus : t.zetaSSigmaPlus;
    return ((e + P) / (s * T)) * t.zetaS0 * crm::exp_cr(d * d / 2.0 * (sig * sig));
  } else if (t.zetaSparam == 5) {
    // a Gaussian bump in T (not in the reference)
    const double x = T - t.zetaSPeakT;
    return t.zetaS0 * crm::exp_cr(-x * x / (2. * t.zetaSWidthT * t.zetaSWidthT));
  }
  return 0.;
}

// TransportCoeff::etaS, src/trancoeff.cpp:73-90
__device__ __forceinline__ double tr_etaS(const TrDev& t, double e, double rho,
                                          double T, double muB, double s, double P) {
  if (t.etaSparam == 0) {
    return t.etaS0;
  } else if (t.etaSparam == 1) {
    return t.etaSMin + ((T > t.T0) ? t.ah * (T - t.T0) : t.al * (T - t.T0));
  } else if (t.etaSparam == 2) {
    return smax(0.0, t.etaSMin + ((e > t.etaSEpsilonMin)
                                      ? ((t.ah * (e - t.etaSEpsilonMin) + t.aRho * rho))
                                      : t.al * (e - t.etaSEpsilonMin) + t.aRho * rho));
  } else if (t.etaSparam == 3) {
    if (!(fabs(s) >= 1.0) || T < 1e-1) return 0;
    const double Tc = t.T0 + t.etaSShiftMuB * (muB / 0.938);
    return ((e + P) / (s * T)) *
           smax(0.0, (t.etaSMin + ((T > Tc) ? t.ah * (T - Tc) : t.al * (T - Tc))) *
                         (1 + t.etaSScaleMuB * (muB / 0.938)));
  }
  return 0.;
}

// TransportCoeff::getTau, src/trancoeff.cpp:92-100.  abs(e + P) binds to
// int abs(int) in the reference: the test is trunc(e + P) != 0.
// etaS and zetaS are tr_etaS and tr_zetaS at the same point (pure
// functions, evaluated once by the caller).
__device__ __forceinline__ void tr_getTau_from(double e, double T, double s, double P,
                                               double etaS, double zetaS, double& taupi,
                                               double& tauPi) {
  if (T > 1e-1 && !(fabs(e + P) < 1.0)) {
    taupi = ddiv((5. / 5.068) * s * etaS, e + P);
    tauPi = ddiv((6. / 5.068) * zetaS * s, e + P);
  } else {
    taupi = tauPi = 0.;
  }
}

__device__ __forceinline__ void tr_getTau(const TrDev& t, double e, double rho,
                                          double T, double muB, double s, double P,
                                          double& taupi, double& tauPi) {
  tr_getTau_from(e, T, s, P, tr_etaS(t, e, rho, T, muB, s, P), tr_zetaS(t, e, T, s, P), taupi,
                 tauPi);
}

// ---------------------------------------------------------- HLLE face flux
// Hydro::hlle_flux, src/hdo.cpp:77-305, for one face given the two
// reconstructed states (L = right edge of the left cell, R = left edge of
// the right cell) and the fill fractions of the two cells in `dir`.
// Returns false when the reference returns without adding a flux.
__device__ __forceinline__ bool hlle_face(int dir, bool predict, double tau, double dt,
                                          double dxdir, Prim l, Prim r, double mL,
                                          double mR, double flux[7], unsigned& err) {
  const double dta = predict ? dt / 2. : dt;
  const double El = ddiv(l.e + l.p, 1 - l.vx * l.vx - l.vy * l.vy - l.vz * l.vz);
  const double Er = ddiv(r.e + r.p, 1 - r.vx * r.vx - r.vy * r.vy - r.vz * r.vz);
  const double tauFactor = predict ? tau + 0.25 * dt : tau + 0.5 * dt;
  if (l.e < 0.) { l.e = 0.; l.p = 0.; }
  if (r.e < 0.) { r.e = 0.; r.p = 0.; }
  if (l.e > 1e10) { err |= ERR_E_HUGE; return false; }
  if (l.e == 0. && r.e == 0.) return false;
  if (mL < 1. && mR < 1.) return false;
  const double cs2 = 1. / 3.;
  const double cs = sqrt(1. / 3.);
  const double gammal = 1. / sqrt(1 - l.vx * l.vx - l.vy * l.vy - l.vz * l.vz);
  const double gammar = 1. / sqrt(1 - r.vx * r.vx - r.vy * r.vy - r.vz * r.vz);
  const double U1l = gammal * gammal * (l.e + l.p) * l.vx;
  const double U2l = gammal * gammal * (l.e + l.p) * l.vy;
  const double U3l = gammal * gammal * (l.e + l.p) * l.vz;
  const double U4l = gammal * gammal * (l.e + l.p) - l.p;
  const double Ubl = gammal * l.nb, Uql = gammal * l.nq, Usl = gammal * l.ns;
  const double U1r = gammar * gammar * (r.e + r.p) * r.vx;
  const double U2r = gammar * gammar * (r.e + r.p) * r.vy;
  const double U3r = gammar * gammar * (r.e + r.p) * r.vz;
  const double U4r = gammar * gammar * (r.e + r.p) - r.p;
  const double Ubr = gammar * r.nb, Uqr = gammar * r.nq, Usr = gammar * r.ns;
  double Ftl, Fxl, Fyl, Fzl, Fbl, Fql, Fsl, Ftr, Fxr, Fyr, Fzr, Fbr, Fqr, Fsr;
  double bl, br;
  const double sEl = sqrtz(El), sEr = sqrtz(Er);
  const double vnl = dir == X_ ? l.vx : (dir == Y_ ? l.vy : l.vz);
  const double vnr = dir == X_ ? r.vx : (dir == Y_ ? r.vy : r.vz);
  if (dir != Z_) {
    Ftl = U4l * vnl + l.p * vnl;
    Fxl = U1l * vnl;
    Fyl = U2l * vnl;
    Fzl = U3l * vnl;
    Fbl = Ubl * vnl; Fql = Uql * vnl; Fsl = Usl * vnl;
    Ftr = U4r * vnr + r.p * vnr;
    Fxr = U1r * vnr;
    Fyr = U2r * vnr;
    Fzr = U3r * vnr;
    Fbr = Ubr * vnr; Fqr = Uqr * vnr; Fsr = Usr * vnr;
    if (dir == X_) { Fxl = Fxl + l.p; Fxr = Fxr + r.p; }
    else { Fyl = Fyl + l.p; Fyr = Fyr + r.p; }
  } else {
    const double tau1 = tauFactor;
    // the 18 quotients by tau1 as one divide-free batch (div_batch)
    double n[18] = {U4l * vnl, l.p * vnl, U1l * vnl, U2l * vnl, U3l * vnl, l.p,
                    Ubl * vnl, Uql * vnl, Usl * vnl,
                    U4r * vnr, r.p * vnr, U1r * vnr, U2r * vnr, U3r * vnr, r.p,
                    Ubr * vnr, Uqr * vnr, Usr * vnr};
    div_batch<18>(n, tau1, 1.0 / tau1, crm::mk_den_ok(tau1));
    Ftl = n[0] + n[1];
    Fxl = n[2];
    Fyl = n[3];
    Fzl = n[4] + n[5];
    Fbl = n[6]; Fql = n[7]; Fsl = n[8];
    Ftr = n[9] + n[10];
    Fxr = n[11];
    Fyr = n[12];
    Fzr = n[13] + n[14];
    Fbr = n[15]; Fqr = n[16]; Fsr = n[17];
  }
  {
    const double ss = sEl + sEr, dv = vnl - vnr;
    const double csb = sqrt(cs2 + ddiv(0.5 * sqrtz(El * Er), ss * ss) * (dv * dv));
    const double vb = ddiv(sEl * vnl + sEr * vnr, sEl + sEr);
    bl = smin(0., smin((vb - csb) / (1 - vb * csb), (vnl - cs) / (1 - vnl * cs)));
    br = smax(0., smax((vb + csb) / (1 + vb * csb), (vnr + cs) / (1 + vnr * cs)));
    if (dir == Z_) {
      bl = 1. / tau * bl;
      br = 1. / tau * br;
      if (l.e == 0.) bl = -1. / tau;
      if (r.e == 0.) br = 1. / tau;
    } else {
      if (l.e == 0.) bl = -1.;
      if (r.e == 0.) br = 1.;
    }
  }
  if (bl == 0. && br == 0.) return false;
  const double pre = tauFactor * dta / dxdir;
  const double den = -bl + br;
  flux[T_] = pre * (-bl * br * (U4l - U4r) + br * Ftl - bl * Ftr);
  flux[X_] = pre * (-bl * br * (U1l - U1r) + br * Fxl - bl * Fxr);
  flux[Y_] = pre * (-bl * br * (U2l - U2r) + br * Fyl - bl * Fyr);
  flux[Z_] = pre * (-bl * br * (U3l - U3r) + br * Fzl - bl * Fzr);
  flux[NB_] = pre * (-bl * br * (Ubl - Ubr) + br * Fbl - bl * Fbr);
  flux[NQ_] = pre * (-bl * br * (Uql - Uqr) + br * Fql - bl * Fqr);
  flux[NS_] = pre * (-bl * br * (Usl - Usr) + br * Fsl - bl * Fsr);
  // divided by den as one divide-free batch (ddiv's results)
  div_batch<7, true>(flux, den, 1.0 / den, crm::mk_den_ok(den));
  if (flux[NB_] != flux[NB_]) { err |= ERR_FLUX_NAN; return false; }
  return true;
}

}  // namespace vh
