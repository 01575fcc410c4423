/*
 * vh_oracle.c -- CPU oracle (test infrastructure only) for the vHLLE
 * per-timestep hydro update.  See vh_oracle.h for the contract.
 *
 * Each function restates the reference function named in its comment, in
 * the reference's own loop and operation order, so that a build with
 * -ffp-contract=off reproduces the reference's FP64 results bit for bit.
 * The restatement is sequential on purpose: the cumulative per-cell flux
 * order it produces (x faces, y faces, z faces, source) is the order the
 * CUDA path has to match.
 */
#include "vh_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { T_ = 0, X_ = 1, Y_ = 2, Z_ = 3, NB_ = 4, NQ_ = 5, NS_ = 6 };
enum { PREDICT = 0, CORRECT = 1 };

int or_abi_version(void) { return 1; }

/* ---------------------------------------------------------------- helpers */

/* minmod slope limiter, src/cll.cpp:12-19 */
/* Fluid's dz (src/fld.cpp:79), or the whole grid's for a slab of it */
static double grid_dz(const or_grid *g) {
  return g->dz > 0. ? g->dz : (g->zmax - g->zmin) / (g->nz - 1);
}

static double minmod(double a, double b) {
  if (a * b <= 0.) return 0.;
  if (fabs(a) > fabs(b))
    return b;
  else
    return a;
}

/* index44, src/cll.cpp:22-31 (indices are always in range here) */
static int index44(int i, int j) {
  if (j < i)
    return (i * (i + 1)) / 2 + j;
  else
    return (j * (j + 1)) / 2 + i;
}

/* std::min / std::max semantics (return the first argument on ties/NaN) */
static double smin(double a, double b) { return (b < a) ? b : a; }
static double smax(double a, double b) { return (a < b) ? b : a; }

/* sign(), src/hdo.cpp:34-41 */
static double sgn(double x) {
  if (x > 0)
    return 1.;
  else if (x < 0.)
    return -1.;
  else
    return 0.;
}

/* ------------------------------------------------------------------- EoS */

/* EoS1f::getue / getun / eos, src/eo1.cpp:63-123 */
static void eos1f(const or_eos *E, double e, double nb, double *T, double *mub,
                  double *p) {
  const int ne = E->ne, nn = E->nn;
  int k, k1, k2;
  k1 = 0;
  k2 = ne - 1;
  while (k2 - k1 > 1) {
    k = (k1 + k2) / 2;
    if (e < E->egrid[k])
      k2 = k;
    else
      k1 = k;
  }
  int ixe = k1;
  if (ixe > ne - 2) ixe = ne - 2;
  const double ue = (e - E->egrid[k1]) / (E->egrid[k2] - E->egrid[k1]);
  k1 = 0;
  k2 = nn - 1;
  while (k2 - k1 > 1) {
    k = (k1 + k2) / 2;
    if (nb < E->ngrid[k])
      k2 = k;
    else
      k1 = k;
  }
  int ixn = k1;
  if (ixn > nn - 2) ixn = nn - 2;
  if (ixn < 0) ixn = 0;
  const double un = (nb - E->ngrid[k1]) / (E->ngrid[k2] - E->ngrid[k1]);
  const double we[2] = {1. - ue, ue};
  const double wn[2] = {1. - un, un};
  double sp = 0., sT = 0., smu = 0.;
  for (int je = 0; je < 2; je++)
    for (int jn = 0; jn < 2; jn++) {
      const int id = (ixe + je) + ne * (ixn + jn);
      sp += we[je] * wn[jn] * E->p[id];
      sT += we[je] * wn[jn] * E->T[id];
      smu += we[je] * wn[jn] * E->mub[id];
    }
  if (sp < 0.) sp = 0.;
  *p = sp;
  *T = sT;
  *mub = smu;
}

/* EoSCMFe's constants, src/eoCMFe.h:10-11 */
#define CMFE_EPS0 (146.51751415742 * 0.87326281)
#define CMFE_N0 (0.15891 * 0.87272727)

/* EoSaux::get, src/eoChiral.cpp:99-130 (EoSaux::p, :132-151, is its p);
 * with cmfe, EoSCMFeaux::get / ::p (src/eoCMFe.cpp:121-189): zeros below
 * EPS_CUTOFF = 2e-2 and a NaN pressure replaced after the interpolation */
static void chiral_aux_x(const or_aux *A, int cmfe, int crmath, double e,
                         double nb, double *p, double *T, double *mub,
                         double *mus) {
  if (cmfe ? e < 2e-2 : e < 0.) {
    *T = *mub = *mus = *p = 0.;
    return;
  }
  const double de = (A->emax - A->emin) / (A->ne - 1);
  const double dn = (A->nmax - A->nmin) / (A->nn - 1);
  int ie = (int)((e - A->emin) / de);
  int in = (int)((nb - A->nmin) / dn);
  if (ie < 0) ie = 0;
  if (in < 0) in = 0;
  if (ie > A->ne - 2) ie = A->ne - 2;
  if (in > A->nn - 2) in = A->nn - 2;
  const double em = e - A->emin - ie * de;
  const double nm = nb - A->nmin - in * dn;
  const double we[2] = {1. - em / de, em / de};
  const double wn[2] = {1. - nm / dn, nm / dn};
  double sp = 0., sT = 0., sb = 0., ss = 0.;
  for (int je = 0; je < 2; je++)
    for (int jn = 0; jn < 2; jn++) {
      const long k = (long)(in + jn) * A->ne + (ie + je);
      sp += we[je] * wn[jn] * A->p[k];
      sT += we[je] * wn[jn] * A->T[k];
      sb += we[je] * wn[jn] * A->mub[k];
      ss += we[je] * wn[jn] * A->mus[k];
    }
  if (cmfe && isnan(sp)) {
    if (e > 0.8 * CMFE_EPS0 || nb > 40. * CMFE_N0) {
      sp = 0.2964 * e;
      sT = 0.15120476935 * (crmath ? or_root4_cr(e) : pow(e, 0.25));
      sb = ss = 0.0;
    } else {
      sT = sb = ss = sp = 0.;
    }
  }
  if (sp < 0.0) sp = 0.0;
  *p = sp;
  *T = sT;
  *mub = sb;
  *mus = ss;
}

static void chiral_aux(const or_aux *A, double e, double nb, double *p,
                       double *T, double *mub, double *mus) {
  chiral_aux_x(A, 0, 0, e, nb, p, T, mub, mus);
}

/* EoSCMFe::eos, src/eoCMFe.cpp:204-217 (muq = 0; ::p, :219-226, is its p) */
static void eos_cmfe(const or_eos *E, double e, double nb, double *T,
                     double *mub, double *mus, double *p) {
  if (e < 15 * CMFE_EPS0 / 1000.0 && nb < 5 * CMFE_N0)
    chiral_aux_x(&E->aux[0], 1, E->crmath, e, nb, p, T, mub, mus);
  else if (e < 0.8 * CMFE_EPS0 && nb < 40. * CMFE_N0)
    chiral_aux_x(&E->aux[1], 1, E->crmath, e, nb, p, T, mub, mus);
  else {
    *p = 0.2964 * e;
    *T = 0.15120476935 * (E->crmath ? or_root4_cr(e) : pow(e, 0.25));
    *mub = *mus = 0.0;
  }
}

/* EoSChiral::eos, src/eoChiral.cpp:159-170 (muq = 0) */
static void eos_chiral(const or_eos *E, double e, double nb, double *T,
                       double *mub, double *mus, double *p) {
  if (e < 1.46 && nb < 0.3)
    chiral_aux(&E->aux[0], e, nb, p, T, mub, mus);
  else if (e < 146. && nb < 6.)
    chiral_aux(&E->aux[1], e, nb, p, T, mub, mus);
  else {
    *p = 0.2964 * e;
    *T = 0.15120476935 * (E->crmath ? or_root4_cr(e) : pow(e, 0.25));
    *mub = *mus = 0.0;
  }
}

/* EoS3f::getue / getun (src/eo3.cpp:98-130): the bracket of the binary
 * search, clamped (the e index only from above), and the weight from the
 * unclamped bracket */
static void eo3_bracket(const double *g, int n, double x, int clamp_low,
                        int *ix, double *u) {
  int k, k1 = 0, k2 = n - 1;
  while (k2 - k1 > 1) {
    k = (k1 + k2) / 2;
    if (x < g[k])
      k2 = k;
    else
      k1 = k;
  }
  *ix = k1;
  if (*ix > n - 2) *ix = n - 2;
  if (clamp_low && *ix < 0) *ix = 0;
  *u = (x - g[k1]) / (g[k2] - g[k1]);
}

/* EoS3f::eos, src/eo3.cpp:132-175.  For e < 0 the reference sets the
 * outputs to 0 and then interpolates anyway (there is no return), so the
 * extrapolated values it computes are what it returns. */
static void eos3f(const or_eos *E, double e, double nb, double nq, double ns,
                  double *T, double *mub, double *muq, double *mus,
                  double *p) {
  const int ne = E->ne, nn = E->nn;
  int ixe, ixnb, ixnq, ixns;
  double ue, ub, uq, us;
  eo3_bracket(E->egrid, ne, e, 0, &ixe, &ue);
  eo3_bracket(E->ngrid, nn, nb, 1, &ixnb, &ub);
  eo3_bracket(E->ngrid, nn, nq, 1, &ixnq, &uq);
  eo3_bracket(E->ngrid, nn, ns, 1, &ixns, &us);
  const double we[2] = {1. - ue, ue}, wnb[2] = {1. - ub, ub};
  const double wnq[2] = {1. - uq, uq}, wns[2] = {1. - us, us};
  double sp = 0., sT = 0., sb = 0., sq = 0., ss = 0.;
  for (int je = 0; je < 2; je++)
    for (int jnb = 0; jnb < 2; jnb++)
      for (int jnq = 0; jnq < 2; jnq++)
        for (int jns = 0; jns < 2; jns++) {
          const long k = (long)(ixe + je) + (long)ne * (ixnb + jnb) +
                         (long)ne * nn * (ixnq + jnq) +
                         (long)ne * nn * nn * (ixns + jns);
          const double w = we[je] * wnb[jnb] * wnq[jnq] * wns[jns];
          sp += w * E->p[k];
          sT += w * E->T[k];
          sb += w * E->mub[k];
          sq += w * E->muq[k];
          ss += w * E->mus[k];
        }
  if (sp < 0.) sp = 0.;
  *p = sp;
  *T = sT;
  *mub = sb;
  *muq = sq;
  *mus = ss;
}

/* EoSHadron: the table position of a charge (the "inverse log mapping" of
 * src/eoHadron.cpp:97-112) */
static double hadron_x(int crmath, double n, double n0, double lognmax,
                       double dxn, double n_abs_min) {
  if (n != 0.0) {
    const double zn = crmath ? or_log_cr(fabs(n) / n0) : log(fabs(n) / n0);
    if (zn >= -lognmax + 2.0 * dxn)
      return n / fabs(n) * 0.5 * (zn + lognmax);
    return n / n_abs_min * dxn;
  }
  return 0.;
}

/* EoSHadron::eos / ::p, src/eoHadron.cpp:81-208 (nq from the caller; the
 * constructor's nb_abs_min, nq_abs_min and e_min recomputed as it does,
 * src/eoHadron.cpp:49-53) */
static void eos_hadron(const or_eos *E, double e, double nb, double nq,
                       double *T, double *mub, double *muq, double *mus,
                       double *p) {
  const int ne = E->hne, nnb = E->hnnb, nnq = E->hnnq;
#define IX3(ie, inb, inq) ((long)(inq) + (long)nnq * (inb) + (long)nnq * nnb * (ie))
  const double dxnb0 = (2.0 * E->lognmax) / (nnb - 1);
  const double dxnq0 = (2.0 * E->lognmax) / (nnq - 1);
  const double nb_abs_min = E->hn0 * exp(2.0 * dxnb0 - E->lognmax);
  const double nq_abs_min = E->hn0 * exp(2.0 * dxnq0 - E->lognmax);
  const double e_min = E->he0 * exp(E->logemin);
  if (e <= 0.) {
    *T = *mub = *muq = *mus = *p = 0.;
    return;
  }
  if (e < e_min) {
    *p = e / e_min * E->p[IX3(0, nnb / 2, nnq / 2)];
    *T = e / e_min * E->T[IX3(0, nnb / 2, nnq / 2)];
    *mub = *muq = *mus = 0.;
    return;
  }
  const double xe = E->crmath ? or_log_cr(e / E->he0) : log(e / E->he0);
  const double dxe = (E->logemax - E->logemin) / (ne - 1);
  const double dxnb = (2.0 * E->lognmax) / (nnb - 1);
  const double dxnq = (2.0 * E->lognmax) / (nnq - 1);
  const double xnb = hadron_x(E->crmath, nb, E->hn0, E->lognmax, dxnb, nb_abs_min);
  const double xnq = hadron_x(E->crmath, nq, E->hn0, E->lognmax, dxnq, nq_abs_min);
  int ie = (int)((xe - E->logemin) / dxe);
  int inb = (int)((xnb + E->lognmax) / dxnb);
  int inq = (int)((xnq + E->lognmax) / dxnq);
  if (ie < 0) ie = 0;
  if (inb < 0) inb = 0;
  if (inq < 0) inq = 0;
  if (ie > ne - 2) ie = ne - 2;
  if (inb > nnb - 2) inb = nnb - 2;
  if (inq > nnq - 2) inq = nnq - 2;
  const double em = xe - E->logemin - ie * dxe;
  const double nbm = xnb + E->lognmax - inb * dxnb;
  const double nqm = xnq + E->lognmax - inq * dxnq;
  if (E->status[IX3(ie, inb, inq)] == 1) {
    *T = *mub = *muq = *mus = *p = 0.;
    return;
  }
  const double we[2] = {1. - em / dxe, em / dxe};
  const double wnb[2] = {1. - nbm / dxnb, nbm / dxnb};
  const double wnq[2] = {1. - nqm / dxnq, nqm / dxnq};
  double sT = 0., sb = 0., sq = 0., ss = 0., sp = 0.;
  for (int je = 0; je < 2; je++)
    for (int jnb = 0; jnb < 2; jnb++)
      for (int jnq = 0; jnq < 2; jnq++) {
        const long k = IX3(ie + je, inb + jnb, inq + jnq);
        sp += we[je] * wnb[jnb] * wnq[jnq] * E->p[k];
        sT += we[je] * wnb[jnb] * wnq[jnq] * E->T[k];
        sb += we[je] * wnb[jnb] * wnq[jnq] * E->mub[k];
        sq += we[je] * wnb[jnb] * wnq[jnq] * E->muq[k];
        ss += we[je] * wnb[jnb] * wnq[jnq] * E->mus[k];
      }
#undef IX3
  if (sp < 0.0) sp = 0.0;
  *p = sp;
  *T = sT;
  *mub = sb;
  *muq = sq;
  *mus = ss;
}

/* EoSSmash::eos / ::p, src/eoSmash.cpp:70-177 */
static void eos_smash(const or_eos *E, double e, double nb, double nq,
                      double *T, double *mub, double *muq, double *mus,
                      double *p) {
  const int ne = E->hne, nnb = E->hnnb, nnq = E->hnnq;
#define IX3(ie, inb, inq) ((long)(inq) + (long)nnq * (inb) + (long)nnq * nnb * (ie))
  if (e <= 0.) {
    *T = *mub = *muq = *mus = *p = 0.;
    return;
  }
  if (e < E->semin) {
    *p = e / E->semin * E->p[IX3(0, nnb / 2, nnq / 2)];
    *T = e / E->semin * E->T[IX3(0, nnb / 2, nnq / 2)];
    *mub = *muq = *mus = 0.;
    return;
  }
  const double de = (E->semax - E->semin) / (ne - 1);
  const double dnb = (E->snbmax - E->snbmin) / (nnb - 1);
  const double dnq = (E->snqmax - E->snqmin) / (nnq - 1);
  int ie = (int)((e - E->semin) / de);
  int inb = (int)((nb - E->snbmin) / dnb);
  int inq = (int)((nq - E->snqmin) / dnq);
  if (ie < 0) ie = 0;
  if (inb < 0) inb = 0;
  if (inq < 0) inq = 0;
  if (ie > ne - 2) ie = ne - 2;
  if (inb > nnb - 2) inb = nnb - 2;
  if (inq > nnq - 2) inq = nnq - 2;
  const double em = e - E->semin - ie * de;
  const double nbm = nb - E->snbmin - inb * dnb;
  const double nqm = nq - E->snqmin - inq * dnq;
  const double we[2] = {1. - em / de, em / de};
  const double wnb[2] = {1. - nbm / dnb, nbm / dnb};
  const double wnq[2] = {1. - nqm / dnq, nqm / dnq};
  double sT = 0., sb = 0., sq = 0., ss = 0., sp = 0.;
  for (int je = 0; je < 2; je++)
    for (int jnb = 0; jnb < 2; jnb++)
      for (int jnq = 0; jnq < 2; jnq++) {
        const long k = IX3(ie + je, inb + jnb, inq + jnq);
        sp += we[je] * wnb[jnb] * wnq[jnq] * E->p[k];
        sT += we[je] * wnb[jnb] * wnq[jnq] * E->T[k];
        sb += we[je] * wnb[jnb] * wnq[jnq] * E->mub[k];
        sq += we[je] * wnb[jnb] * wnq[jnq] * E->muq[k];
        ss += we[je] * wnb[jnb] * wnq[jnq] * E->mus[k];
      }
#undef IX3
  if (sp < 0.0) sp = 0.0;
  *p = sp;
  *T = sT;
  *mub = sb;
  *muq = sq;
  *mus = ss;
}

/* EoSAZHaux::get, src/eoAZH.cpp:58-83 */
static double azh_get(const struct or_azh *t, double e, double nb) {
  if (e <= 0.) return 0.0;
  int ie = (int)((e - t->emin) / t->de);
  int in = (int)((nb - t->nmin) / t->dn);
  if (ie < 0) ie = 0;
  if (in < 0) in = 0;
  if (ie > t->ne - 2) ie = t->ne - 2;
  if (in > t->nn - 2) in = t->nn - 2;
  const double em = (e - t->emin - ie * t->de) / t->de;
  const double nm = (nb - t->nmin - in * t->dn) / t->dn;
  const double we[2] = {1. - em, em};
  const double wn[2] = {1. - nm, nm};
  double value = 0.0;
  for (int je = 0; je < 2; je++)
    for (int jn = 0; jn < 2; jn++)
      value += we[je] * wn[jn] * t->v[(long)(ie + je) * t->nn + (in + jn)];
  return value;
}

/* EoSAZHaux::getLow, src/eoAZH.cpp:85-102 (its exit for nb beyond 10000
 * cells left out: the clamped cell extrapolates) */
static double azh_low(const struct or_azh *t, double e, double nb) {
  if (e <= 0.) return 0.0;
  int in = (int)((nb - t->nmin) / t->dn);
  if (in < 0) in = 0;
  if (in > t->nn - 2) in = t->nn - 2;
  const double nm = (nb - t->nmin - in * t->dn) / t->dn;
  const double wn[2] = {1. - nm, nm};
  const double value = wn[0] * t->v[in] + wn[1] * t->v[in + 1];
  return value * e / t->emin;
}

/* EoSAZH::eos, src/eoAZH.cpp:123-140 (p, T at |nb|, muB at nb) */
static void eos_azh(const or_eos *E, double e, double nb, double *T,
                    double *mub, double *p) {
  const struct or_azh *a = E->az;
  const double anb = fabs(nb);
  if (e > a[0].emin + a[0].de * (a[0].ne - 1)) {
    *p = azh_get(&a[1], e, anb);
    *T = azh_get(&a[3], e, anb);
    *mub = azh_get(&a[5], e, nb);
  } else if (e > a[0].emin) {
    *p = azh_get(&a[0], e, anb);
    *T = azh_get(&a[2], e, anb);
    *mub = azh_get(&a[4], e, nb);
  } else {
    *p = azh_low(&a[0], e, anb);
    *T = azh_low(&a[2], e, anb);
    *mub = azh_low(&a[4], e, nb);
  }
}

/* EoS::eos() with muq; muq = 0 but for kind 3, mus = 0 but for kinds 2, 3 */
static void eos_eval5(const or_eos *E, double e, double nb, double *T,
                      double *mub, double *muq, double *mus, double *p) {
  *muq = 0.;
  if (E->kind == 3) {
    eos3f(E, e, nb, 0., 0., T, mub, muq, mus, p);
    return;
  }
  if (E->kind == 4) {
    eos_hadron(E, e, nb, 0., T, mub, muq, mus, p);
    return;
  }
  if (E->kind == 5) {
    eos_smash(E, e, nb, 0., T, mub, muq, mus, p);
    return;
  }
  *mus = 0.;
  if (E->kind == 0) {
    *p = e / 3.;
    *T = e > 0. ? sqrt(sqrt(e / E->conf_cnst)) : 0.;
    *mub = 0.;
  } else if (E->kind == 2) {
    eos_chiral(E, e, nb, T, mub, mus, p);
  } else if (E->kind == 6) {
    eos_azh(E, e, nb, T, mub, p);
  } else if (E->kind == 7) {
    eos_cmfe(E, e, nb, T, mub, mus, p);
  } else {
    eos1f(E, e, nb, T, mub, p);
  }
}

static void eos_eval4(const or_eos *E, double e, double nb, double *T,
                      double *mub, double *mus, double *p) {
  double muq;
  eos_eval5(E, e, nb, T, mub, &muq, mus, p);
}

static void eos_eval(const or_eos *E, double e, double nb, double *T,
                     double *mub, double *p) {
  double mus;
  eos_eval4(E, e, nb, T, mub, &mus, p);
}

/* EoS::p; EoSChiral::p (src/eoChiral.cpp:172-178) is its eos's p */
static double eos_p(const or_eos *E, double e, double nb) {
  double T, mub, mus, p;
  if (E->kind == 0) return e / 3.;
  if (E->kind == 3) {
    double muq;
    eos3f(E, e, nb, 0., 0., &T, &mub, &muq, &mus, &p);
    return p;
  }
  if (E->kind == 4) {
    double muq;
    eos_hadron(E, e, nb, 0., &T, &mub, &muq, &mus, &p);
    return p;
  }
  if (E->kind == 5) {
    double muq;
    eos_smash(E, e, nb, 0., &T, &mub, &muq, &mus, &p);
    return p;
  }
  if (E->kind == 2) {
    eos_chiral(E, e, nb, &T, &mub, &mus, &p);
    return p;
  }
  if (E->kind == 7) {
    eos_cmfe(E, e, nb, &T, &mub, &mus, &p);
    return p;
  }
  if (E->kind == 6) {  /* EoSAZH::p, src/eoAZH.cpp:142-150: eos's p */
    eos_azh(E, e, nb, &T, &mub, &p);
    return p;
  }
  eos1f(E, e, nb, &T, &mub, &p);
  return p;
}

/* EoS::s, src/eos.cpp:18-25 */
static double eos_s(const or_eos *E, double e, double nb, double nq,
                    double ns) {
  double T, mub, mus, p, muq;
  eos_eval5(E, e, nb, &T, &mub, &muq, &mus, &p);
  if (T > 0.0)
    return (e + p - mub * nb - muq * nq - mus * ns) / T;
  else
    return 0.;
}

/* ------------------------------------------------------- transformPV */

/* transformPV, src/rmn.cpp:28-139.  Q is modified in place exactly as the
 * reference does when |M| > Q_t (the caller's copy). */
static void transform_pv(const or_eos *E, double Q[7], double *e, double *p,
                         double *nb, double *nq, double *ns, double *vx,
                         double *vy, double *vz) {
  const int MAXIT = 100;
  const double dpe = 1. / 3.;
  const double corrf = 0.9999;
  double v, vl = 0., vh = 1., dvold, dv, f, df;
  double M = sqrt(Q[X_] * Q[X_] + Q[Y_] * Q[Y_] + Q[Z_] * Q[Z_]);
  if (Q[T_] <= 0.) {
    *e = 0.;
    *p = 0.;
    *vx = *vy = *vz = 0.;
    *nb = *nq = *ns = 0.;
    return;
  }
  if (M == 0.) {
    *e = Q[T_];
    *vx = 0.;
    *vy = 0.;
    *vz = 0.;
    *nb = Q[NB_];
    *nq = Q[NQ_];
    *ns = Q[NS_];
    *p = eos_p(E, *e, *nb);
    return;
  }
  if (M > Q[T_]) {
    Q[X_] *= corrf * Q[T_] / M;
    Q[Y_] *= corrf * Q[T_] / M;
    Q[Z_] *= corrf * Q[T_] / M;
    M = Q[T_] * corrf;
  }
  v = 0.5 * (vl + vh);
  *e = Q[T_] - M * v;
  if (*e < 0.) *e = 0.;
  *nb = Q[NB_] * sqrt(1 - v * v);
  *nq = Q[NQ_] * sqrt(1 - v * v);
  *ns = Q[NS_] * sqrt(1 - v * v);
  *p = eos_p(E, *e, *nb);
  f = (Q[T_] + *p) * v - M;
  df = (Q[T_] + *p) - M * v * dpe;
  dvold = vh - vl;
  dv = dvold;
  for (int i = 0; i < MAXIT; i++) {
    if ((f + df * (vh - v)) * (f + df * (vl - v)) >= 0. ||
        fabs(2. * f) > fabs(dvold * df)) {
      dvold = dv;
      dv = 0.5 * (vh - vl);
      v = vl + dv;
    } else {
      dvold = dv;
      dv = f / df;
      v -= dv;
    }
    if (fabs(dv) < (E->tol > 0. ? E->tol : 0.00001)) break;
    *e = Q[T_] - M * v;
    if (*e < 0.) *e = 0.;
    *nb = Q[NB_] * sqrt(1 - v * v);
    *nq = Q[NQ_] * sqrt(1 - v * v);
    *ns = Q[NS_] * sqrt(1 - v * v);
    *p = eos_p(E, *e, *nb);
    f = (Q[T_] + *p) * v - M;
    df = (Q[T_] + *p) - M * v * dpe;
    if (f > 0.)
      vh = v;
    else
      vl = v;
  }
  *vx = v * Q[X_] / M;
  *vy = v * Q[Y_] / M;
  *vz = v * Q[Z_] / M;
  *e = Q[T_] - M * v;
  *p = eos_p(E, *e, *nb); /* stale nb, as in the reference */
  *nb = Q[NB_] * sqrt(1 - *vx * *vx - *vy * *vy - *vz * *vz);
  *nq = Q[NQ_] * sqrt(1 - *vx * *vx - *vy * *vy - *vz * *vz);
  *ns = Q[NS_] * sqrt(1 - *vx * *vx - *vy * *vy - *vz * *vz);
}

/* ------------------------------------------------ transport coefficients */

/* TransportCoeff::zetaS, src/trancoeff.cpp:19-66.  cs2(e) is the EoS base
 * class value 1/3 for both supported EoS kinds (src/eos.h:37). */
#define TR_EXP(x) (t->crmath ? or_exp_cr(x) : exp(x))
#define TR_ROOT4(x) (t->crmath ? or_root4_cr(x) : pow((x), 0.25))
static double tr_zetaS(const or_trc *t, double e, double T, double s,
                       double P) {
  const double cs2e = 1. / 3.;
  const double T_p = 0.180, T_peak = 0.165, T_width = 0.010, B_norm = 0.24,
               B_width = 1.5, T_peak2 = 0.160, B_norm2 = 0.13, B1 = 0.01,
               B2 = 0.12;
  if (t->zetaSparam == 0)
    return t->zetaS0 * (1. / 3. - cs2e) / (TR_EXP((0.16 - T) / 0.001) + 1.);
  else if (t->zetaSparam == 1) {
    if (T < 0.180)
      return 0.03 + (0.08 * TR_EXP(((T / T_p) - 1.) / (0.0025))) +
             (0.22 * TR_EXP(((T / T_p) - 1) / (0.022)));
    else if (T >= 0.180 && T < 0.200)
      return 27.55 * (T / T_p) - 13.45 - (13.77 * (T / T_p) * (T / T_p));
    else if (T >= 0.200)
      return 0.001 + (0.9 * TR_EXP(-((T / T_p) - 1.) / (0.0025))) +
             (0.25 * TR_EXP(-((T / T_p) - 1.) / (0.13)));
  } else if (t->zetaSparam == 2) {
    if (T > T_peak)
      return B_norm * ((B_width * B_width) /
                       ((((T / T_peak) - 1.) * ((T / T_peak) - 1.)) +
                        (B_width * B_width)));
    else if (T <= T_peak)
      return B_norm *
             (TR_EXP(-((T - T_peak) / T_width) * ((T - T_peak) / T_width)));
  } else if (t->zetaSparam == 3) {
    if (T < T_peak2)
      return B_norm2 * TR_EXP(-((T - T_peak2) * (T - T_peak2) / (B1 * B1)));
    else if (T >= T_peak2)
      return B_norm2 * TR_EXP(-((T - T_peak2) * (T - T_peak2) / (B2 * B2)));
  } else if (t->zetaSparam == 4) {
    /* abs() binds to int abs(int) in the reference: |s| < 1 reads as 0 */
    if (!(fabs(s) >= 1.0) || T < 1e-1) return 0;
    const double d =
        t->zetaSScaleBeta * (TR_ROOT4(e) - TR_ROOT4(t->zetaSPeakEpsilon));
    const double sig =
        e < t->zetaSPeakEpsilon ? t->zetaSSigmaMinus : t->zetaSSigmaPlus;
    return ((e + P) / (s * T)) * t->zetaS0 * TR_EXP(d * d / 2.0 * (sig * sig));
  } else if (t->zetaSparam == 5) {
    /* a Gaussian bump in T: not in the reference */
    const double x = T - t->zetaSPeakT;
    return t->zetaS0 * TR_EXP(-x * x / (2. * t->zetaSWidthT * t->zetaSWidthT));
  }
  return 0.;
}

/* TransportCoeff::etaS, src/trancoeff.cpp:73-90 */
static double tr_etaS(const or_trc *t, double e, double rho, double T,
                      double muB, double s, double P) {
  if (t->etaSparam == 0) {
    return t->etaS0;
  } else if (t->etaSparam == 1) {
    return t->etaSMin + ((T > t->T0) ? t->ah * (T - t->T0) : t->al * (T - t->T0));
  } else if (t->etaSparam == 2) {
    return smax(0.0, t->etaSMin + ((e > t->etaSEpsilonMin)
                                       ? ((t->ah * (e - t->etaSEpsilonMin) +
                                           t->aRho * rho))
                                       : t->al * (e - t->etaSEpsilonMin) +
                                             t->aRho * rho));
  } else if (t->etaSparam == 3) {
    if (!(fabs(s) >= 1.0) || T < 1e-1) return 0;
    const double Tc = t->T0 + t->etaSShiftMuB * (muB / 0.938);
    return ((e + P) / (s * T)) *
           smax(0.0, (t->etaSMin + ((T > Tc) ? t->ah * (T - Tc)
                                             : t->al * (T - Tc))) *
                         (1 + t->etaSScaleMuB * (muB / 0.938)));
  }
  return 0.;
}

/* TransportCoeff::getTau, src/trancoeff.cpp:92-100.  The reference's
 * abs(e + P) resolves to int abs(int): the test is trunc(e + P) != 0. */
static void tr_getTau(const or_trc *t, double e, double rho, double T,
                      double muB, double s, double P, double *taupi,
                      double *tauPi) {
  if (T > 1e-1 && !(fabs(e + P) < 1.0)) {
    *taupi = (5. / 5.068) * s * tr_etaS(t, e, rho, T, muB, s, P) / (e + P);
    *tauPi = (6. / 5.068) * tr_zetaS(t, e, T, s, P) * s / (e + P);
  } else {
    *taupi = *tauPi = 0.;
  }
}

static int tr_isViscous(const or_trc *t) {
  return (t->etaS0 > 0. || t->zetaS0 > 0. || t->etaSparam > 0 ||
          t->zetaSparam > 0);
}

/* ------------------------------------------------------------ the step */

typedef struct Ctx {
  const or_grid *g;
  const or_eos *E;
  const or_trc *tr;
  or_state *s;
  long N;
  int nx, ny, nz;
  double dx, dy, dz;
  double tau, dt;
  double *flux, *dm, *pi0, *piH0, *Pi0, *PiH0;
  int err;
} Ctx;

static long cell(const Ctx *c, int ix, int iy, int iz) {
  ix = ix > 0 ? ix : 0;
  ix = ix < c->nx ? ix : c->nx - 1;
  iy = iy > 0 ? iy : 0;
  iy = iy < c->ny ? iy : c->ny - 1;
  iz = iz > 0 ? iz : 0;
  iz = iz < c->nz ? iz : c->nz - 1;
  return (long)ix + (long)c->nx * iy + (long)c->nx * c->ny * iz;
}

static void coords(const Ctx *c, long i, int *ix, int *iy, int *iz) {
  *ix = (int)(i % c->nx);
  *iy = (int)((i / c->nx) % c->ny);
  *iz = (int)(i / ((long)c->nx * c->ny));
}

static long neighbour(const Ctx *c, long i, int dir, int step) {
  int ix, iy, iz;
  coords(c, i, &ix, &iy, &iz);
  if (dir == X_) ix += step;
  if (dir == Y_) iy += step;
  if (dir == Z_) iz += step;
  return cell(c, ix, iy, iz);
}

#define F(a, comp, i) ((a)[(long)(comp) * c->N + (i)])

static double getM(const Ctx *c, long i, int dir) {
  return c->s->m[(long)(dir - 1) * c->N + i];
}
static double getMaxM(const Ctx *c, long i) {
  const double *m = c->s->m;
  return smax(m[i], smax(m[c->N + i], m[2 * c->N + i]));
}

static void addFlux(Ctx *c, long i, const double f[7]) {
  for (int k = 0; k < 7; k++) F(c->flux, k, i) += f[k];
}

/* Cell::getPrimVar / getPrimVarHCenter / getPrimVarPrev,
 * src/cll.cpp:90-104,206-220: con2prim of (field / tau) */
static void primCenter(Ctx *c, const double *field, long i, double tau,
                       double *e, double *p, double *nb, double *nq,
                       double *ns, double *vx, double *vy, double *vz) {
  double q[7];
  for (int k = 0; k < 7; k++) q[k] = F(field, k, i) / tau;
  transform_pv(c->E, q, e, p, nb, nq, ns, vx, vy, vz);
}

/* getPrimVarLeft/Right and the H variants, src/cll.cpp:106-204.
 * side = -1: left boundary of cell i; +1: right boundary. */
static void primFace(Ctx *c, const double *field, long i, int dir, int side,
                     double tau, double *e, double *p, double *nb, double *nq,
                     double *ns, double *vx, double *vy, double *vz) {
  const long inext = neighbour(c, i, dir, +1), iprev = neighbour(c, i, dir, -1);
  double Qr[7], Ql[7], Q[7], dQ[7], q[7];
  for (int k = 0; k < 7; k++) {
    Qr[k] = F(field, k, inext);
    Ql[k] = F(field, k, iprev);
    Q[k] = F(field, k, i);
  }
  for (int k = 0; k < 7; k++)
    dQ[k] = minmod((Qr[k] - Q[k]) / 2., (Q[k] - Ql[k]) / 2.);
  if (side < 0)
    for (int k = 0; k < 7; k++) q[k] = (Q[k] - dQ[k]) / tau;
  else
    for (int k = 0; k < 7; k++) q[k] = (Q[k] + dQ[k]) / tau;
  transform_pv(c->E, q, e, p, nb, nq, ns, vx, vy, vz);
}

/* Hydro::hlle_flux, src/hdo.cpp:77-305 */
static void hlle_flux(Ctx *c, long L, long R, int direction, int mode) {
  double el, er, pl, pr, nbl, nql, nsl, nbr, nqr, nsr, vxl, vxr, vyl, vyr, vzl,
      vzr, bl = 0., br = 0., csb, vb, El, Er, dx = 0.;
  double Ftl = 0., Fxl = 0., Fyl = 0., Fzl = 0., Fbl = 0., Fql = 0., Fsl = 0.,
         Ftr = 0., Fxr = 0., Fyr = 0., Fzr = 0., Fbr = 0., Fqr = 0., Fsr = 0.;
  double U1l, U2l, U3l, U4l, Ubl, Uql, Usl, U1r, U2r, U3r, U4r, Ubr, Uqr, Usr;
  double flux[7];
  const double dt = c->dt, tau = c->tau;
  const double dta = mode == 0 ? dt / 2. : dt;
  double tauFactor;
  const double *QQ = (mode == PREDICT) ? c->s->Q : c->s->Qh;
  primFace(c, QQ, L, direction, +1, tau, &el, &pl, &nbl, &nql, &nsl, &vxl,
           &vyl, &vzl);
  primFace(c, QQ, R, direction, -1, tau, &er, &pr, &nbr, &nqr, &nsr, &vxr,
           &vyr, &vzr);
  El = (el + pl) / (1 - vxl * vxl - vyl * vyl - vzl * vzl);
  Er = (er + pr) / (1 - vxr * vxr - vyr * vyr - vzr * vzr);
  if (mode == PREDICT)
    tauFactor = tau + 0.25 * dt;
  else
    tauFactor = tau + 0.5 * dt;

  if (el < 0.) {
    el = 0.;
    pl = 0.;
  }
  if (er < 0.) {
    er = 0.;
    pr = 0.;
  }
  if (el > 1e10) { /* the reference dumps the cell and exits */
    c->err |= OR_ERR_E_HUGE;
    return;
  }
  if (el == 0. && er == 0.) return;
  /* pr < 0: the reference re-evaluates the same two calls; no effect */
  if (getM(c, L, direction) < 1. && getM(c, R, direction) < 1.) return;

  const double cs2 = 1. / 3.;
  const double cs = sqrt(1. / 3.);
  double gammal = 1. / sqrt(1 - vxl * vxl - vyl * vyl - vzl * vzl);
  double gammar = 1. / sqrt(1 - vxr * vxr - vyr * vyr - vzr * vzr);
  U1l = gammal * gammal * (el + pl) * vxl;
  U2l = gammal * gammal * (el + pl) * vyl;
  U3l = gammal * gammal * (el + pl) * vzl;
  U4l = gammal * gammal * (el + pl) - pl;
  Ubl = gammal * nbl;
  Uql = gammal * nql;
  Usl = gammal * nsl;
  U1r = gammar * gammar * (er + pr) * vxr;
  U2r = gammar * gammar * (er + pr) * vyr;
  U3r = gammar * gammar * (er + pr) * vzr;
  U4r = gammar * gammar * (er + pr) - pr;
  Ubr = gammar * nbr;
  Uqr = gammar * nqr;
  Usr = gammar * nsr;

  const double sEl = sqrt(El), sEr = sqrt(Er);
  if (direction == X_) {
    Ftl = U4l * vxl + pl * vxl;
    Fxl = U1l * vxl + pl;
    Fyl = U2l * vxl;
    Fzl = U3l * vxl;
    Fbl = Ubl * vxl;
    Fql = Uql * vxl;
    Fsl = Usl * vxl;
    Ftr = U4r * vxr + pr * vxr;
    Fxr = U1r * vxr + pr;
    Fyr = U2r * vxr;
    Fzr = U3r * vxr;
    Fbr = Ubr * vxr;
    Fqr = Uqr * vxr;
    Fsr = Usr * vxr;
    const double ss = sEl + sEr, dv = vxl - vxr;
    csb = sqrt(cs2 + 0.5 * sqrt(El * Er) / (ss * ss) * (dv * dv));
    vb = (sEl * vxl + sEr * vxr) / (sEl + sEr);
    bl = smin(0., smin((vb - csb) / (1 - vb * csb), (vxl - cs) / (1 - vxl * cs)));
    br = smax(0., smax((vb + csb) / (1 + vb * csb), (vxr + cs) / (1 + vxr * cs)));
    dx = c->dx;
    if (el == 0.) bl = -1.;
    if (er == 0.) br = 1.;
  }
  if (direction == Y_) {
    Ftl = U4l * vyl + pl * vyl;
    Fxl = U1l * vyl;
    Fyl = U2l * vyl + pl;
    Fzl = U3l * vyl;
    Fbl = Ubl * vyl;
    Fql = Uql * vyl;
    Fsl = Usl * vyl;
    Ftr = U4r * vyr + pr * vyr;
    Fxr = U1r * vyr;
    Fyr = U2r * vyr + pr;
    Fzr = U3r * vyr;
    Fbr = Ubr * vyr;
    Fqr = Uqr * vyr;
    Fsr = Usr * vyr;
    const double ss = sEl + sEr, dv = vyl - vyr;
    csb = sqrt(cs2 + 0.5 * sqrt(El * Er) / (ss * ss) * (dv * dv));
    vb = (sEl * vyl + sEr * vyr) / (sEl + sEr);
    bl = smin(0., smin((vb - csb) / (1 - vb * csb), (vyl - cs) / (1 - vyl * cs)));
    br = smax(0., smax((vb + csb) / (1 + vb * csb), (vyr + cs) / (1 + vyr * cs)));
    dx = c->dy;
    if (el == 0.) bl = -1.;
    if (er == 0.) br = 1.;
  }
  if (direction == Z_) {
    const double tau1 = tauFactor;
    Ftl = U4l * vzl / tau1 + pl * vzl / tau1;
    Fxl = U1l * vzl / tau1;
    Fyl = U2l * vzl / tau1;
    Fzl = U3l * vzl / tau1 + pl / tau1;
    Fbl = Ubl * vzl / tau1;
    Fql = Uql * vzl / tau1;
    Fsl = Usl * vzl / tau1;
    Ftr = U4r * vzr / tau1 + pr * vzr / tau1;
    Fxr = U1r * vzr / tau1;
    Fyr = U2r * vzr / tau1;
    Fzr = U3r * vzr / tau1 + pr / tau1;
    Fbr = Ubr * vzr / tau1;
    Fqr = Uqr * vzr / tau1;
    Fsr = Usr * vzr / tau1;
    const double ss = sEl + sEr, dv = vzl - vzr;
    csb = sqrt(cs2 + 0.5 * sqrt(El * Er) / (ss * ss) * (dv * dv));
    vb = (sEl * vzl + sEr * vzr) / (sEl + sEr);
    bl = 1. / tau *
         smin(0., smin((vb - csb) / (1 - vb * csb), (vzl - cs) / (1 - vzl * cs)));
    br = 1. / tau *
         smax(0., smax((vb + csb) / (1 + vb * csb), (vzr + cs) / (1 + vzr * cs)));
    dx = c->dz;
    if (el == 0.) bl = -1. / tau;
    if (er == 0.) br = 1. / tau;
  }
  if (bl == 0. && br == 0.) return;

  flux[T_] = tauFactor * dta / dx *
             (-bl * br * (U4l - U4r) + br * Ftl - bl * Ftr) / (-bl + br);
  flux[X_] = tauFactor * dta / dx *
             (-bl * br * (U1l - U1r) + br * Fxl - bl * Fxr) / (-bl + br);
  flux[Y_] = tauFactor * dta / dx *
             (-bl * br * (U2l - U2r) + br * Fyl - bl * Fyr) / (-bl + br);
  flux[Z_] = tauFactor * dta / dx *
             (-bl * br * (U3l - U3r) + br * Fzl - bl * Fzr) / (-bl + br);
  flux[NB_] = tauFactor * dta / dx *
              (-bl * br * (Ubl - Ubr) + br * Fbl - bl * Fbr) / (-bl + br);
  flux[NQ_] = tauFactor * dta / dx *
              (-bl * br * (Uql - Uqr) + br * Fql - bl * Fqr) / (-bl + br);
  flux[NS_] = tauFactor * dta / dx *
              (-bl * br * (Usl - Usr) + br * Fsl - bl * Fsr) / (-bl + br);
  if (flux[NB_] != flux[NB_]) {
    c->err |= OR_ERR_FLUX_NAN;
    return;
  }
  double mf[7];
  for (int k = 0; k < 7; k++) mf[k] = -flux[k];
  addFlux(c, L, mf);
  addFlux(c, R, flux);
}

/* Hydro::source + source_step, src/hdo.cpp:307-353 */
static void source_step(Ctx *c, long i, int mode) {
  const double dt = c->dt, tau = c->tau;
  const double _dt = (mode == PREDICT) ? dt / 2. : dt;
  double tau1, Q[7], k[7], _Q[7];
  const double *field = (mode == PREDICT) ? c->s->Q : c->s->Qh;
  for (int j = 0; j < 7; j++) Q[j] = F(field, j, i);
  tau1 = (mode == PREDICT) ? tau : tau + 0.5 * dt;
  double e, p, nb, nq, ns, vx, vy, vz;
  for (int j = 0; j < 7; j++) _Q[j] = Q[j] / tau1;
  transform_pv(c->E, _Q, &e, &p, &nb, &nq, &ns, &vx, &vy, &vz);
  k[T_] = -_Q[T_] * vz * vz - p * (1. + vz * vz);
  k[X_] = 0.;
  k[Y_] = 0.;
  k[Z_] = -_Q[Z_];
  k[NB_] = 0.;
  k[NQ_] = 0.;
  k[NS_] = 0.;
  for (int j = 0; j < 7; j++) k[j] *= _dt;
  if (k[NB_] != k[NB_]) {
    c->err |= OR_ERR_SOURCE_NAN;
    return;
  }
  addFlux(c, i, k);
}

/* Cell::setQ / setQh zeroing copy, src/cll.h:75-86 (Q) */
static void copyQ(Ctx *c, double *field, long dst, long src) {
  double q[7];
  for (int k = 0; k < 7; k++) q[k] = F(field, k, src);
  if (q[T_] < 0.)
    for (int k = 0; k < 7; k++) q[k] = 0.;
  for (int k = 0; k < 7; k++) F(field, k, dst) = q[k];
}

static void copyVisc(Ctx *c, long dst, long src) {
  double p[10];
  for (int k = 0; k < 10; k++) p[k] = F(c->s->pi, k, src);
  const double P = c->s->Pi[src];
  for (int k = 0; k < 10; k++) F(c->s->pi, k, dst) = p[k];
  c->s->Pi[dst] = P;
}

/* Fluid::correctImagCells (full = 0) and correctImagCellsFull (full = 1),
 * src/fld.cpp:211-382 */
static void correctImagCells(Ctx *c, int full) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  double *Q = c->s->Q, *Qh = c->s->Qh;
  /* Z */
  for (int ix = 0; ix < nx; ix++)
    for (int iy = 0; iy < ny; iy++) {
      long s = cell(c, ix, iy, 2);
      copyQ(c, Q, cell(c, ix, iy, 1), s);
      copyQ(c, Q, cell(c, ix, iy, 0), s);
      if (!full) {
        copyQ(c, Qh, cell(c, ix, iy, 1), s);
        copyQ(c, Qh, cell(c, ix, iy, 0), s);
      } else {
        double p[10];
        for (int k = 0; k < 10; k++) p[k] = F(c->s->pi, k, s);
        const double P = c->s->Pi[s];
        long d0 = cell(c, ix, iy, 0), d1 = cell(c, ix, iy, 1);
        for (int k = 0; k < 10; k++) F(c->s->pi, k, d0) = p[k];
        for (int k = 0; k < 10; k++) F(c->s->pi, k, d1) = p[k];
        c->s->Pi[d0] = P;
        c->s->Pi[d1] = P;
      }
      s = cell(c, ix, iy, nz - 3);
      copyQ(c, Q, cell(c, ix, iy, nz - 2), s);
      copyQ(c, Q, cell(c, ix, iy, nz - 1), s);
      if (!full) {
        copyQ(c, Qh, cell(c, ix, iy, nz - 2), s);
        copyQ(c, Qh, cell(c, ix, iy, nz - 1), s);
      } else {
        double p[10];
        for (int k = 0; k < 10; k++) p[k] = F(c->s->pi, k, s);
        const double P = c->s->Pi[s];
        long d0 = cell(c, ix, iy, nz - 2), d1 = cell(c, ix, iy, nz - 1);
        for (int k = 0; k < 10; k++) F(c->s->pi, k, d0) = p[k];
        for (int k = 0; k < 10; k++) F(c->s->pi, k, d1) = p[k];
        c->s->Pi[d0] = P;
        c->s->Pi[d1] = P;
      }
    }
  /* Y */
  for (int ix = 0; ix < nx; ix++)
    for (int iz = 0; iz < nz; iz++) {
      long s = cell(c, ix, 2, iz);
      copyQ(c, Q, cell(c, ix, 1, iz), s);
      copyQ(c, Q, cell(c, ix, 0, iz), s);
      if (!full) {
        copyQ(c, Qh, cell(c, ix, 1, iz), s);
        copyQ(c, Qh, cell(c, ix, 0, iz), s);
      } else {
        copyVisc(c, cell(c, ix, 0, iz), s);
        copyVisc(c, cell(c, ix, 1, iz), s);
      }
      s = cell(c, ix, ny - 3, iz);
      copyQ(c, Q, cell(c, ix, ny - 2, iz), s);
      copyQ(c, Q, cell(c, ix, ny - 1, iz), s);
      if (!full) {
        copyQ(c, Qh, cell(c, ix, ny - 2, iz), s);
        copyQ(c, Qh, cell(c, ix, ny - 1, iz), s);
      } else {
        copyVisc(c, cell(c, ix, ny - 2, iz), s);
        copyVisc(c, cell(c, ix, ny - 1, iz), s);
      }
    }
  /* X */
  for (int iy = 0; iy < ny; iy++)
    for (int iz = 0; iz < nz; iz++) {
      long s = cell(c, 2, iy, iz);
      copyQ(c, Q, cell(c, 1, iy, iz), s);
      copyQ(c, Q, cell(c, 0, iy, iz), s);
      if (!full) {
        copyQ(c, Qh, cell(c, 1, iy, iz), s);
        copyQ(c, Qh, cell(c, 0, iy, iz), s);
      } else {
        copyVisc(c, cell(c, 0, iy, iz), s);
        copyVisc(c, cell(c, 1, iy, iz), s);
      }
      s = cell(c, nx - 3, iy, iz);
      copyQ(c, Q, cell(c, nx - 2, iy, iz), s);
      copyQ(c, Q, cell(c, nx - 1, iy, iz), s);
      if (!full) {
        copyQ(c, Qh, cell(c, nx - 2, iy, iz), s);
        copyQ(c, Qh, cell(c, nx - 1, iy, iz), s);
      } else {
        copyVisc(c, cell(c, nx - 2, iy, iz), s);
        copyVisc(c, cell(c, nx - 1, iy, iz), s);
      }
    }
}

/* Cell::addM, src/cll.h:147-151 */
static void addM(Ctx *c, long i, int dir, double inc) {
  double *m = c->s->m;
  m[(long)(dir - 1) * c->N + i] += inc;
  if (m[(long)(dir - 1) * c->N + i] > 0.9)
    for (int k = 0; k < 3; k++) m[(long)k * c->N + i] = 1.;
}

/* Fluid::updateM, src/fld.cpp:384-423 */
static void updateM(Ctx *c, double tau, double dt) {
  const long N = c->N;
  double *dm = c->dm;
  for (int ix = 0; ix < c->nx; ix++)
    for (int iy = 0; iy < c->ny; iy++)
      for (int iz = 0; iz < c->nz; iz++) {
        const long i = cell(c, ix, iy, iz);
        dm[i] = dm[N + i] = dm[2 * N + i] = 0.;
        if (getMaxM(c, i) < 1.) {
          if (getM(c, cell(c, ix + 1, iy, iz), X_) >= 1. ||
              getM(c, cell(c, ix - 1, iy, iz), X_) >= 1.)
            dm[i] = dt / c->dx;
          if (getM(c, cell(c, ix, iy + 1, iz), Y_) >= 1. ||
              getM(c, cell(c, ix, iy - 1, iz), Y_) >= 1.)
            dm[N + i] = dt / c->dy;
          if (getM(c, cell(c, ix, iy, iz + 1), Z_) >= 1. ||
              getM(c, cell(c, ix, iy, iz - 1), Z_) >= 1.)
            dm[2 * N + i] = dt / c->dz / tau;
          if (dm[i] == 0. && dm[N + i] == 0.) {
            if (getMaxM(c, cell(c, ix + 1, iy + 1, iz)) >= 1. ||
                getMaxM(c, cell(c, ix + 1, iy - 1, iz)) >= 1. ||
                getMaxM(c, cell(c, ix - 1, iy + 1, iz)) >= 1. ||
                getMaxM(c, cell(c, ix - 1, iy - 1, iz)) >= 1.) {
              dm[i] = 0.707 * dt / c->dx;
              dm[N + i] = 0.707 * dt / c->dy;
            }
          }
        }
      }
  for (int ix = 0; ix < c->nx; ix++)
    for (int iy = 0; iy < c->ny; iy++)
      for (int iz = 0; iz < c->nz; iz++) {
        const long i = cell(c, ix, iy, iz);
        addM(c, i, X_, dm[i]);
        addM(c, i, Y_, dm[N + i]);
        addM(c, i, Z_, dm[2 * N + i]);
      }
}

static double getpi(const Ctx *c, const double *a, long i, int mu, int nu) {
  return a[(long)index44(mu, nu) * c->N + i];
}

/* Hydro::NSquant, src/hdo.cpp:381-652.  M is ISformal's one dbeta matrix
 * (NULL with vorticity off): rows are written only where the reference
 * writes them, and nothing next to vacuum, so the rest keeps the values of
 * earlier cells. */
static void NSquant(Ctx *c, int ix, int iy, int iz, double pi[4][4],
                    double *Pi, double dmu[4][4], double (*M)[4], double *du) {
  const double VMIN = 1e-2;
  const double UDIFF = 3.0;
  const double tau = c->tau, dt = c->dt;
  double e0, e1, p, nb, nq, ns, vx1, vy1, vz1, vx0, vy0, vz0, vxH, vyH, vzH;
  double T, mub, T0 = 0., T1 = 0.;
  double ut0, ux0, uy0, uz0, ut1, ux1, uy1, uz1;
  double uuu[4];
  const double gmunu[4][4] = {
      {1, 0, 0, 0}, {0, -1, 0, 0}, {0, 0, -1, 0}, {0, 0, 0, -1}};
  const long ic = cell(c, ix, iy, iz);
  const double dx = c->dx, dy = c->dy, dz = c->dz;
  if (getMaxM(c, cell(c, ix + 1, iy, iz)) <= 0.9 ||
      getMaxM(c, cell(c, ix, iy + 1, iz)) <= 0.9 ||
      getMaxM(c, cell(c, ix - 1, iy, iz)) <= 0.9 ||
      getMaxM(c, cell(c, ix, iy - 1, iz)) <= 0.9 ||
      getMaxM(c, cell(c, ix + 1, iy + 1, iz)) <= 0.9 ||
      getMaxM(c, cell(c, ix + 1, iy - 1, iz)) <= 0.9 ||
      getMaxM(c, cell(c, ix - 1, iy + 1, iz)) <= 0.9 ||
      getMaxM(c, cell(c, ix - 1, iy - 1, iz)) <= 0.9) {
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        pi[i][j] = 0.;
        dmu[i][j] = 0.;
      }
    *Pi = *du = 0.;
    return;
  }
  primCenter(c, c->s->Qprev, ic, tau - dt, &e0, &p, &nb, &nq, &ns, &vx0, &vy0,
             &vz0);
  if (M) eos_eval(c->E, e0, nb, &T0, &mub, &p);
  primCenter(c, c->s->Q, ic, tau, &e1, &p, &nb, &nq, &ns, &vx1, &vy1, &vz1);
  if (M) eos_eval(c->E, e1, nb, &T1, &mub, &p);
  primCenter(c, c->s->Qh, ic, tau - 0.5 * dt, &e1, &p, &nb, &nq, &ns, &vxH,
             &vyH, &vzH);
  double etaS, zetaS;
  double s = eos_s(c->E, e1, nb, nq, ns);
  eos_eval(c->E, e1, nb, &T, &mub, &p);
  etaS = tr_etaS(c->tr, e1, nb, T, mub, s, p);
  zetaS = tr_zetaS(c->tr, e1, T, s, p);
  ut0 = 1.0 / sqrt(1.0 - vx0 * vx0 - vy0 * vy0 - vz0 * vz0);
  ux0 = ut0 * vx0;
  uy0 = ut0 * vy0;
  uz0 = ut0 * vz0;
  ut1 = 1.0 / sqrt(1.0 - vx1 * vx1 - vy1 * vy1 - vz1 * vz1);
  ux1 = ut1 * vx1;
  uy1 = ut1 * vy1;
  uz1 = ut1 * vz1;
  uuu[0] = 1.0 / sqrt(1.0 - vxH * vxH - vyH * vyH - vzH * vzH);
  uuu[1] = uuu[0] * vxH;
  uuu[2] = uuu[0] * vyH;
  uuu[3] = uuu[0] * vzH;

  dmu[0][0] = (ut1 * ut1 - ut0 * ut0) / 2. / uuu[0] / dt;
  dmu[0][1] = (ux1 * ux1 - ux0 * ux0) / 2. / uuu[1] / dt;
  dmu[0][2] = (uy1 * uy1 - uy0 * uy0) / 2. / uuu[2] / dt;
  dmu[0][3] = (uz1 * uz1 - uz0 * uz0) / 2. / uuu[3] / dt;
  if (M) { /* src/hdo.cpp:450-459; e1 is the half-step centre's here */
    M[0][0] = (ut1 / T1 - ut0 / T0) / dt;
    M[0][1] = (ux1 / T1 - ux0 / T0) / dt;
    M[0][2] = (uy1 / T1 - uy0 / T0) / dt;
    M[0][3] = (uz1 / T1 - uz0 / T0) / dt;
    if (e1 <= 0. || e0 <= 0. || T1 <= 0. || T0 <= 0.)
      M[0][0] = M[0][1] = M[0][2] = M[0][3] = 0.;
  }
  if (fabs(0.5 * (ut1 + ut0) / ut1) > UDIFF) dmu[0][0] = (ut1 - ut0) / dt;
  if (fabs(uuu[1]) < VMIN || fabs(0.5 * (ux1 + ux0) / ux1) > UDIFF)
    dmu[0][1] = (ux1 - ux0) / dt;
  if (fabs(uuu[2]) < VMIN || fabs(0.5 * (uy1 + uy0) / uy1) > UDIFF)
    dmu[0][2] = (uy1 - uy0) / dt;
  if (fabs(uuu[3]) < VMIN || fabs(0.5 * (uz1 + uz0) / uz1) > UDIFF)
    dmu[0][3] = (uz1 - uz0) / dt;
  if (e1 <= 0. || e0 <= 0.) {
    dmu[0][0] = dmu[0][1] = dmu[0][2] = dmu[0][3] = 0.;
  }
  /* spatial derivatives: d = 1 (x), 2 (y), 3 (eta) */
  for (int d = 1; d <= 3; d++) {
    long ip, im;
    if (d == 1) {
      ip = cell(c, ix + 1, iy, iz);
      im = cell(c, ix - 1, iy, iz);
    } else if (d == 2) {
      ip = cell(c, ix, iy + 1, iz);
      im = cell(c, ix, iy - 1, iz);
    } else {
      ip = cell(c, ix, iy, iz + 1);
      im = cell(c, ix, iy, iz - 1);
    }
    primCenter(c, c->s->Qh, ip, tau, &e1, &p, &nb, &nq, &ns, &vx1, &vy1, &vz1);
    if (M) eos_eval(c->E, e1, nb, &T1, &mub, &p);
    primCenter(c, c->s->Qh, im, tau, &e0, &p, &nb, &nq, &ns, &vx0, &vy0, &vz0);
    if (M) eos_eval(c->E, e0, nb, &T0, &mub, &p);
    if (e1 > 0. && e0 > 0.) {
      ut0 = 1.0 / sqrt(1.0 - vx0 * vx0 - vy0 * vy0 - vz0 * vz0);
      ux0 = ut0 * vx0;
      uy0 = ut0 * vy0;
      uz0 = ut0 * vz0;
      ut1 = 1.0 / sqrt(1.0 - vx1 * vx1 - vy1 * vy1 - vz1 * vz1);
      ux1 = ut1 * vx1;
      uy1 = ut1 * vy1;
      uz1 = ut1 * vz1;
      if (M) { /* src/hdo.cpp:491-500, 537-546, 583-592 */
        const double h = d == 1 ? dx : d == 2 ? dy : dz * (tau + 0.5 * dt);
        M[d][0] = 0.5 * (ut1 / T1 - ut0 / T0) / h;
        M[d][1] = 0.5 * (ux1 / T1 - ux0 / T0) / h;
        M[d][2] = 0.5 * (uy1 / T1 - uy0 / T0) / h;
        M[d][3] = 0.5 * (uz1 / T1 - uz0 / T0) / h;
        if (e1 <= 0. || e0 <= 0. || T1 <= 0. || T0 <= 0.)
          M[d][0] = M[d][1] = M[d][2] = M[d][3] = 0.;
      }
      if (d == 1 || d == 2) {
        const double h = (d == 1) ? dx : dy;
        dmu[d][0] = 0.25 * (ut1 * ut1 - ut0 * ut0) / uuu[0] / h;
        dmu[d][1] = 0.25 * (ux1 * ux1 - ux0 * ux0) / uuu[1] / h;
        dmu[d][2] = 0.25 * (uy1 * uy1 - uy0 * uy0) / uuu[2] / h;
        dmu[d][3] = 0.25 * (uz1 * uz1 - uz0 * uz0) / uuu[3] / h;
        if (fabs(0.5 * (ut1 + ut0) / uuu[0]) > UDIFF)
          dmu[d][0] = 0.5 * (ut1 - ut0) / h;
        if (fabs(uuu[1]) < VMIN || fabs(0.5 * (ux1 + ux0) / uuu[1]) > UDIFF)
          dmu[d][1] = 0.5 * (ux1 - ux0) / h;
        if (fabs(uuu[2]) < VMIN || fabs(0.5 * (uy1 + uy0) / uuu[2]) > UDIFF)
          dmu[d][2] = 0.5 * (uy1 - uy0) / h;
        if (fabs(uuu[3]) < VMIN || fabs(0.5 * (uz1 + uz0) / uuu[3]) > UDIFF)
          dmu[d][3] = 0.5 * (uz1 - uz0) / h;
      } else {
        const double th = tau + 0.5 * dt;
        dmu[3][0] = 0.25 * (ut1 * ut1 - ut0 * ut0) / uuu[0] / dz / th;
        dmu[3][1] = 0.25 * (ux1 * ux1 - ux0 * ux0) / uuu[1] / dz / th;
        dmu[3][2] = 0.25 * (uy1 * uy1 - uy0 * uy0) / uuu[2] / dz / th;
        dmu[3][3] = 0.25 * (uz1 * uz1 - uz0 * uz0) / uuu[3] / dz / th;
        if (fabs(0.5 * (ut1 + ut0) / uuu[0]) > UDIFF)
          dmu[3][0] = 0.5 * (ut1 - ut0) / dz / th;
        if (fabs(uuu[1]) < VMIN || fabs(0.5 * (ux1 + ux0) / uuu[1]) > UDIFF)
          dmu[3][1] = 0.5 * (ux1 - ux0) / dz / th;
        if (fabs(uuu[2]) < VMIN || fabs(0.5 * (uy1 + uy0) / uuu[2]) > UDIFF)
          dmu[3][2] = 0.5 * (uy1 - uy0) / dz / th;
        if (fabs(uuu[3]) < VMIN || fabs(0.5 * (uz1 + uz0) / uuu[3]) > UDIFF)
          dmu[3][3] = 0.5 * (uz1 - uz0) / dz / th;
      }
    } else {
      dmu[d][0] = dmu[d][1] = dmu[d][2] = dmu[d][3] = 0.;
    }
  }
  dmu[3][0] += uuu[3] / (tau - 0.5 * dt);
  dmu[3][3] += uuu[0] / (tau - 0.5 * dt);
  if (M && T > 0.) { /* src/hdo.cpp:608-611 */
    M[3][0] += uuu[3] / (T * (tau - 0.5 * dt));
    M[3][3] += uuu[0] / (T * (tau - 0.5 * dt));
  }
  /* Z^{mu nu lambda rho} contraction, element by element */
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double acc = 0.0;
      for (int k = 0; k < 4; k++)
        for (int l = 0; l < 4; l++) {
          double Z = 0.0;
          if (j == l) Z += 0.5 * (gmunu[i][k] - uuu[i] * uuu[k]);
          if (i == l) Z += 0.5 * (gmunu[j][k] - uuu[j] * uuu[k]);
          if (k == l) Z -= (gmunu[i][j] - uuu[i] * uuu[j]) / 3.0;
          acc += Z * dmu[k][l] * 2.0 * etaS * s / 5.068;
        }
      pi[i][j] = acc;
    }
  *Pi = -zetaS * s * (dmu[0][0] + dmu[1][1] + dmu[2][2] + dmu[3][3]) / 5.068;
  *du = dmu[0][0] + dmu[1][1] + dmu[2][2] + dmu[3][3];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      if (isinf(pi[i][j]) || isnan(pi[i][j])) c->err |= OR_ERR_NSQUANT_NAN;
}

/* Hydro::ISformal, src/hdo.cpp:682-963 (first-order relaxation, no
 * FORMAL_SOLUTION).  With vorticity (s->dbeta set) one dbeta matrix, zero
 * at the start of the call, goes through NSquant cell after cell in loop
 * order; each cell with matter stores it clamped (Cell::setDbeta,
 * src/cll.h:173-183), each empty cell stores zeros (Cell::resetDbeta). */
static void ISformal(Ctx *c) {
  const double tau = c->tau, dt = c->dt;
  const double gmumu[4] = {1., -1., -1., -1.};
  const long N = c->N;
  double *dbeta = c->s->dbeta;
  double Mb[4][4] = {{0.}};
  double (*M)[4] = dbeta ? Mb : NULL;
  double *pi0 = c->pi0, *piH0 = c->piH0, *Pi0 = c->Pi0, *PiH0 = c->PiH0;
  const double *cpi = c->s->pi;
  const double *cPi = c->s->Pi;
#define PI(i, j) cpi[(long)index44(i, j) * N + ic]
#define PIH0(i, j) piH0[(long)index44(i, j) * N + ic]
#define PI0(i, j) pi0[(long)index44(i, j) * N + ic]
  /* loop #1 */
  for (int ix = 0; ix < c->nx; ix++)
    for (int iy = 0; iy < c->ny; iy++)
      for (int iz = 0; iz < c->nz; iz++) {
        const long ic = cell(c, ix, iy, iz);
        double e, p, nb, nq, ns, vx, vy, vz, T, mub;
        double piNS[4][4], sigNS[4][4], PiNS, dmu[4][4], du;
        primCenter(c, c->s->Qh, ic, tau - dt / 2., &e, &p, &nb, &nq, &ns, &vx,
                   &vy, &vz);
        if (e <= 0.) {
          for (int i = 0; i < 4; i++)
            for (int j = 0; j <= i; j++) {
              PIH0(i, j) = 0.0;
              PI0(i, j) = 0.0;
            }
          PiH0[ic] = 0.0;
          Pi0[ic] = 0.0;
          if (dbeta)
            for (int k = 0; k < 16; k++) dbeta[(long)k * N + ic] = 0.0;
          continue;
        }
        double gamma = 1.0 / sqrt(1.0 - vx * vx - vy * vy - vz * vz);
        double u[4];
        u[0] = gamma;
        u[1] = u[0] * vx;
        u[2] = u[0] * vy;
        u[3] = u[0] * vz;
        double flux[7] = {0., 0., 0., 0., 0., 0., 0.};
        for (int i = 0; i < 4; i++)
          flux[i] = (tau - dt) * (PI(0, i) + cPi[ic] * u[0] * u[i]);
        flux[0] += -(tau - dt) * cPi[ic];
        addFlux(c, ic, flux);
        NSquant(c, ix, iy, iz, piNS, &PiNS, dmu, M, &du);
        if (dbeta)
          for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++)
              dbeta[(long)(4 * a + b) * N + ic] = smax(smin(M[a][b], 100.), -100.);
        eos_eval(c->E, e, nb, &T, &mub, &p);
        double etaS, zetaS;
        const double s = eos_s(c->E, e, nb, nq, ns);
        etaS = tr_etaS(c->tr, e, nb, T, mub, s, p);
        zetaS = tr_zetaS(c->tr, e, T, s, p);
        (void)zetaS;
        const double eta = etaS * s;
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++) {
            sigNS[i][j] = 0.5 * piNS[i][j] / eta * 5.068;
            if (eta <= 0.0) sigNS[i][j] = 0.0;
          }
        double taupi, tauPi;
        tr_getTau(c->tr, e, nb, T, mub, s, p, &taupi, &tauPi);
        double deltapipi, taupipi, lambdapiPi, phi7, delPiPi, lamPipi;
        /* TransportCoeff::getOther / getOtherBulk, src/trancoeff.h:28-37 */
        deltapipi = 4. / 3.;
        taupipi = 10. / 7.;
        lambdapiPi = 6. / 5.;
        phi7 = 9. / 70. / eos_p(c->E, e, nb);
        if (isinf(phi7)) phi7 = 0.0;
        phi7 = phi7 / taupi;
        if (taupi < 0.5 * dt) deltapipi = taupipi = lambdapiPi = phi7 = 0.0;
        delPiPi = 2. / 3.;
        lamPipi = 8. / 5. * (1. / 3. - 1. / 3.);
        if (tauPi < 0.5 * dt) delPiPi = lamPipi = 0.0;
        double Delta[10];
        for (int i = 0; i < 4; i++)
          for (int j = 0; j <= i; j++) {
            Delta[index44(i, j)] = -u[i] * u[j];
            if (i == j) Delta[index44(i, j)] += gmumu[i];
            if (taupi > 0.5 * dt)
              PIH0(i, j) = PI(i, j) - (PI(i, j) - piNS[i][j]) * dt / 2.0 /
                                          gamma / taupi;
            else
              PIH0(i, j) = piNS[i][j];
          }
        if (tauPi > 0.5 * dt)
          PiH0[ic] = cPi[ic] - (cPi[ic] - PiNS) * dt / 2.0 / gamma / tauPi;
        else
          PiH0[ic] = PiNS;
        double tau1 = tau - dt * 0.75;
        PIH0(0, 0) += -2. * vz * PI(0, 3) / tau1 * dt / 2.;
        PIH0(3, 3) += -(2. * vz / tau1 * PI(0, 3)) * dt / 2.;
        PIH0(3, 0) += -(vz / tau1 * PI(0, 0) + vz / tau1 * PI(3, 3)) * dt / 2.;
        PIH0(1, 0) += -vz / tau1 * PI(1, 3) * dt / 2.;
        PIH0(2, 0) += -vz / tau1 * PI(2, 3) * dt / 2.;
        PIH0(3, 1) += -(vz / tau1 * PI(0, 1)) * dt / 2.;
        PIH0(3, 2) += -(vz / tau1 * PI(0, 2)) * dt / 2.;
        for (int i = 0; i < 4; i++)
          for (int j = 0; j <= i; j++) {
            PIH0(i, j) += (-deltapipi * PI(i, j) * du +
                           lambdapiPi * cPi[ic] * sigNS[i][j]) /
                          gamma * 0.5 * dt;
            for (int k = 0; k < 4; k++) {
              PIH0(i, j) += (phi7 * PI(i, k) * PI(j, k) * gmumu[k] -
                             taupipi * 0.5 *
                                 (PI(i, k) * sigNS[j][k] * gmumu[k] +
                                  PI(j, k) * sigNS[i][k] * gmumu[k])) /
                            gamma * 0.5 * dt;
              for (int l = 0; l < 4; l++) {
                PIH0(i, j) +=
                    (-PI(i, k) * u[j] - PI(j, k) * u[i]) * u[l] * dmu[l][k] *
                        gmumu[k] / gamma * 0.5 * dt -
                    1. / 3. * Delta[index44(i, j)] * PI(k, l) *
                        (phi7 * PI(k, l) - taupipi * sigNS[k][l]) * gmumu[k] *
                        gmumu[l] / gamma * 0.5 * dt;
              }
            }
          }
        for (int k = 0; k < 4; k++)
          for (int l = 0; l < 4; l++)
            PiH0[ic] += lamPipi * PI(k, l) * sigNS[k][l] * gmumu[k] *
                        gmumu[l] / gamma * 0.5 * dt;
        PiH0[ic] += -delPiPi * cPi[ic] * du / gamma * 0.5 * dt;
        for (int i = 0; i < 4; i++)
          for (int j = 0; j <= i; j++) {
            if (taupi > 0.5 * dt)
              PI0(i, j) =
                  PI(i, j) - (PIH0(i, j) - piNS[i][j]) * dt / gamma / taupi;
            else
              PI0(i, j) = piNS[i][j];
          }
        if (tauPi > 0.5 * dt)
          Pi0[ic] = cPi[ic] - (PiH0[ic] - PiNS) * dt / gamma / tauPi;
        else
          Pi0[ic] = PiNS;
        tau1 = tau - dt * 0.5;
        PI0(0, 0) += -2. * vz / tau1 * PIH0(0, 3) * dt;
        PI0(3, 3) += -(2. * vz / tau1 * PIH0(0, 3)) * dt;
        PI0(3, 0) += -(vz / tau1 * PIH0(0, 0) + vz / tau1 * PIH0(3, 3)) * dt;
        PI0(1, 0) += -vz / tau1 * PIH0(1, 3) * dt;
        PI0(2, 0) += -vz / tau1 * PIH0(2, 3) * dt;
        PI0(3, 1) += -(vz / tau1 * PIH0(0, 1)) * dt;
        PI0(3, 2) += -(vz / tau1 * PIH0(0, 2)) * dt;
        for (int i = 0; i < 4; i++)
          for (int j = 0; j <= i; j++) {
            PI0(i, j) += (-deltapipi * PIH0(i, j) * du +
                          lambdapiPi * PiH0[ic] * sigNS[i][j]) /
                         gamma * dt;
            for (int k = 0; k < 4; k++) {
              PI0(i, j) += (phi7 * PI(i, k) * PIH0(j, k) * gmumu[k] -
                            taupipi * 0.5 *
                                (PIH0(i, k) * sigNS[j][k] * gmumu[k] +
                                 PIH0(j, k) * sigNS[i][k] * gmumu[k])) /
                           gamma * dt;
              for (int l = 0; l < 4; l++) {
                PI0(i, j) +=
                    ((-PIH0(i, k) * u[j] - PIH0(j, k) * u[i]) * u[l] *
                         dmu[l][k] * gmumu[k] -
                     1. / 3. * Delta[index44(i, j)] * PIH0(k, l) *
                         (phi7 * PIH0(k, l) - taupipi * sigNS[k][l]) *
                         gmumu[k] * gmumu[l]) /
                    gamma * dt;
              }
            }
          }
        for (int k = 0; k < 4; k++)
          for (int l = 0; l < 4; l++)
            Pi0[ic] += lamPipi * PIH0(k, l) * sigNS[k][l] * gmumu[k] *
                       gmumu[l] / gamma * dt;
        Pi0[ic] += -delPiPi * PiH0[ic] * du / gamma * dt;
      }
#undef PI
#undef PIH0
#undef PI0

  /* loop #2: advection, limiter, -(tau)*delta Q_{n+1} source */
  double *spi = c->s->pi, *spiH = c->s->piH, *sPi = c->s->Pi,
         *sPiH = c->s->PiH;
  for (int ix = 0; ix < c->nx; ix++)
    for (int iy = 0; iy < c->ny; iy++)
      for (int iz = 0; iz < c->nz; iz++) {
        const long ic = cell(c, ix, iy, iz);
        double e, p, nb, nq, ns, vx, vy, vz;
        double pi[4][4], piH[4][4], Pi, PiH;
        primCenter(c, c->s->Qh, ic, tau - 0.5 * dt, &e, &p, &nb, &nq, &ns, &vx,
                   &vy, &vz);
        if (e <= 0.) continue;
        double xm = -vx * dt / c->dx;
        double ym = -vy * dt / c->dy;
        double zm = -vz * dt / c->dz / (tau - 0.5 * dt);
        double xmH = -vx * dt / c->dx / 2.0;
        double ymH = -vy * dt / c->dy / 2.0;
        double zmH = -vz * dt / c->dz / (tau - 0.5 * dt) / 2.0;
        double wx[2] = {(1. - fabs(xm)), fabs(xm)};
        double wy[2] = {(1. - fabs(ym)), fabs(ym)};
        double wz[2] = {(1. - fabs(zm)), fabs(zm)};
        double wxH[2] = {(1. - fabs(xmH)), fabs(xmH)};
        double wyH[2] = {(1. - fabs(ymH)), fabs(ymH)};
        double wzH[2] = {(1. - fabs(zmH)), fabs(zmH)};
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++) pi[i][j] = piH[i][j] = 0.0;
        Pi = PiH = 0.0;
        for (int jx = 0; jx < 2; jx++)
          for (int jy = 0; jy < 2; jy++)
            for (int jz = 0; jz < 2; jz++) {
              const long c1 =
                  cell(c, (int)(ix + jx * sgn(xm)), (int)(iy + jy * sgn(ym)),
                       (int)(iz + jz * sgn(zm)));
              for (int i = 0; i < 4; i++)
                for (int j = 0; j < 4; j++) {
                  pi[i][j] += wx[jx] * wy[jy] * wz[jz] *
                              pi0[(long)index44(i, j) * N + c1];
                  piH[i][j] += wxH[jx] * wyH[jy] * wzH[jz] *
                               piH0[(long)index44(i, j) * N + c1];
                }
              Pi += wx[jx] * wy[jy] * wz[jz] * Pi0[c1];
              PiH += wxH[jx] * wyH[jy] * wzH[jz] * PiH0[c1];
            }
        double maxT0 = smax((e + p) / (1. - vx * vx - vy * vy - vz * vz) - p,
                            (e + p) * (vx * vx + vy * vy + vz * vz) /
                                    (1. - vx * vx - vy * vy - vz * vz) +
                                p);
        double maxpi = 0.;
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++)
            if (fabs(pi[i][j]) > maxpi) maxpi = fabs(pi[i][j]);
        int rescaled = 0;
        if (maxT0 / maxpi < 1.0) {
          for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) {
              pi[i][j] = 0.1 * pi[i][j] * maxT0 / maxpi;
              piH[i][j] = 0.1 * piH[i][j] * maxT0 / maxpi;
            }
          rescaled = 1;
        }
        if (fabs(Pi) > p) {
          if (Pi != 0.) Pi = 1 * Pi / fabs(Pi) * p;
          if (PiH != 0.) PiH = 1 * PiH / fabs(PiH) * p;
          rescaled = 1;
        }
        c->s->vcc[ic] = rescaled ? maxT0 / maxpi : 1.;
        for (int i = 0; i < 4; i++)
          for (int j = 0; j <= i; j++) {
            spi[(long)index44(i, j) * N + ic] = pi[i][j];
            spiH[(long)index44(i, j) * N + ic] = piH[i][j];
          }
        sPi[ic] = Pi;
        sPiH[ic] = PiH;
        double gamma = 1.0 / sqrt(1.0 - vx * vx - vy * vy - vz * vz);
        double u[4];
        u[0] = gamma;
        u[1] = u[0] * vx;
        u[2] = u[0] * vy;
        u[3] = u[0] * vz;
        double flux[7] = {0., 0., 0., 0., 0., 0., 0.};
        for (int i = 0; i < 4; i++)
          flux[i] = -tau * (getpi(c, spi, ic, 0, i) + sPi[ic] * u[0] * u[i]);
        flux[0] += tau * sPi[ic];
        addFlux(c, ic, flux);
      }
}

/* Hydro::visc_flux, src/hdo.cpp:966-1014 */
static void visc_flux(Ctx *c, long L, long R, int direction) {
  const double tau = c->tau, dt = c->dt;
  double flux[4];
  int ind2 = 0;
  double dxa = 0.;
  if (getM(c, L, direction) < 1. && getM(c, R, direction) < 1.) return;
  if (direction == X_)
    dxa = c->dx;
  else if (direction == Y_)
    dxa = c->dy;
  else if (direction == Z_)
    dxa = c->dz * (tau + 0.5 * dt);
  double e, p, nb, nq, ns, vxl, vyl, vzl, vxr, vyr, vzr;
  primCenter(c, c->s->Qh, L, tau - dt / 2., &e, &p, &nb, &nq, &ns, &vxl, &vyl,
             &vzl);
  primCenter(c, c->s->Qh, R, tau - dt / 2., &e, &p, &nb, &nq, &ns, &vxr, &vyr,
             &vzr);
  vxl = 0.5 * (vxl + vxr);
  vyl = 0.5 * (vyl + vyr);
  vzl = 0.5 * (vzl + vzr);
  double v = sqrt(vxl * vxl + vyl * vyl + vzl * vzl);
  if (v > 1.) {
    vxl = 0.99 * vxl / v;
    vyl = 0.99 * vyl / v;
    vzl = 0.99 * vzl / v;
  }
  double gamma = 1. / sqrt(1. - v * v);
  double uuu[4] = {gamma, gamma * vxl, gamma * vyl, gamma * vzl};
  const double gmumu[4] = {1., -1., -1., -1.};
  ind2 = direction;
  const double *piH = c->s->piH, *PiH = c->s->PiH;
  for (int ind1 = 0; ind1 < 4; ind1++) {
    flux[ind1] = 0.5 * (getpi(c, piH, L, ind1, ind2) + getpi(c, piH, R, ind1, ind2));
    if (ind1 == ind2) flux[ind1] += -0.5 * (PiH[L] + PiH[R]) * gmumu[ind1];
    flux[ind1] += 0.5 * (PiH[L] + PiH[R]) * uuu[ind1] * uuu[ind2];
  }
  for (int i = 0; i < 4; i++) flux[i] = flux[i] * (tau - 0.5 * dt) * dt / dxa;
  double fl[7] = {-flux[0], -flux[1], -flux[2], -flux[3], 0., 0., 0.};
  double fr[7] = {flux[0], flux[1], flux[2], flux[3], 0., 0., 0.};
  addFlux(c, L, fl);
  addFlux(c, R, fr);
}

/* Hydro::visc_source_step, src/hdo.cpp:355-375 */
static void visc_source_step(Ctx *c, long i) {
  const double tau = c->tau, dt = c->dt;
  double e, p, nb, nq, ns, vx, vy, vz, uuu[4], k[7];
  primCenter(c, c->s->Qh, i, tau - dt / 2., &e, &p, &nb, &nq, &ns, &vx, &vy,
             &vz);
  if (e <= 0.) return;
  uuu[0] = 1. / sqrt(1. - vx * vx - vy * vy - vz * vz);
  uuu[1] = uuu[0] * vx;
  uuu[2] = uuu[0] * vy;
  uuu[3] = uuu[0] * vz;
  const double piH33 = getpi(c, c->s->piH, i, 3, 3);
  const double piH03 = getpi(c, c->s->piH, i, 0, 3);
  const double PiH = c->s->PiH[i];
  k[T_] = -piH33 + PiH * (-1.0 - uuu[3] * uuu[3]);
  k[X_] = 0.;
  k[Y_] = 0.;
  k[Z_] = -(piH03 + PiH * uuu[0] * uuu[3]);
  for (int j = 0; j < 4; j++) k[j] *= dt;
  k[NB_] = k[NQ_] = k[NS_] = 0.;
  addFlux(c, i, k);
}

/* Cell::updateByViscFlux, src/cll.cpp:76-84 */
static void updateByViscFlux(Ctx *c, long i) {
  double *Q = c->s->Q;
  const double q0 = F(Q, 0, i), f0 = F(c->flux, 0, i);
  if (fabs(f0) <= 0.5 * q0) {
    for (int k = 0; k < 7; k++) F(Q, k, i) += F(c->flux, k, i);
  } else if (f0 != 0.) {
    const double fac = fabs(0.5 * q0 / f0);
    for (int k = 0; k < 7; k++) F(Q, k, i) += fac * F(c->flux, k, i);
  }
}

static void clearFlux(Ctx *c, long i) {
  for (int k = 0; k < 7; k++) F(c->flux, k, i) = 0.;
}

/* Hydro::performStep, src/hdo.cpp:1016-1134 */
int or_step(const or_grid *g, const or_eos *eos, const or_trc *tr,
            or_state *s, double *tau, double dt) {
  Ctx cx;
  Ctx *c = &cx;
  memset(c, 0, sizeof(*c));
  c->g = g;
  c->E = eos;
  c->tr = tr;
  c->s = s;
  c->nx = g->nx;
  c->ny = g->ny;
  c->nz = g->nz;
  c->N = (long)g->nx * g->ny * g->nz;
  c->dx = (g->xmax - g->xmin) / (g->nx - 1);
  c->dy = (g->ymax - g->ymin) / (g->ny - 1);
  c->dz = grid_dz(g);
  c->tau = *tau;
  c->dt = dt;
  const long N = c->N;
  c->flux = (double *)calloc((size_t)(7 * N), sizeof(double));
  c->dm = (double *)calloc((size_t)(3 * N), sizeof(double));
  c->pi0 = (double *)calloc((size_t)(10 * N), sizeof(double));
  c->piH0 = (double *)calloc((size_t)(10 * N), sizeof(double));
  c->Pi0 = (double *)calloc((size_t)N, sizeof(double));
  c->PiH0 = (double *)calloc((size_t)N, sizeof(double));
  const int nx = c->nx, ny = c->ny, nz = c->nz;

  updateM(c, c->tau, dt);

  /* predictor */
  for (long i = 0; i < N; i++) {
    for (int k = 0; k < 7; k++) F(s->Qprev, k, i) = F(s->Q, k, i);
    clearFlux(c, i);
  }
  for (int mode = PREDICT; mode <= CORRECT; mode++) {
    for (int iy = 0; iy < ny; iy++)
      for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx - 1; ix++)
          hlle_flux(c, cell(c, ix, iy, iz), cell(c, ix + 1, iy, iz), X_, mode);
    for (int iz = 0; iz < nz; iz++)
      for (int ix = 0; ix < nx; ix++)
        for (int iy = 0; iy < ny - 1; iy++)
          hlle_flux(c, cell(c, ix, iy, iz), cell(c, ix, iy + 1, iz), Y_, mode);
    for (int ix = 0; ix < nx; ix++)
      for (int iy = 0; iy < ny; iy++)
        for (int iz = 0; iz < nz - 1; iz++)
          hlle_flux(c, cell(c, ix, iy, iz), cell(c, ix, iy, iz + 1), Z_, mode);
    for (int iy = 0; iy < ny; iy++)
      for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++) {
          const long i = cell(c, ix, iy, iz);
          source_step(c, i, mode);
          if (mode == PREDICT) {
            /* Cell::updateQtoQhByFlux, src/cll.cpp:86-88 */
            for (int k = 0; k < 7; k++)
              F(s->Qh, k, i) = F(s->Q, k, i) + F(c->flux, k, i);
          } else {
            /* Cell::updateByFlux, src/cll.cpp:70-74 */
            if (!(F(s->Q, 0, i) + F(c->flux, 0, i) < 0.))
              for (int k = 0; k < 7; k++) F(s->Q, k, i) += F(c->flux, k, i);
          }
          clearFlux(c, i);
        }
  }
  c->tau += dt;
  correctImagCells(c, 0);

  if (tr_isViscous(tr)) {
    ISformal(c);
    for (int iy = 0; iy < ny; iy++)
      for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx - 1; ix++)
          visc_flux(c, cell(c, ix, iy, iz), cell(c, ix + 1, iy, iz), X_);
    for (int iz = 0; iz < nz; iz++)
      for (int ix = 0; ix < nx; ix++)
        for (int iy = 0; iy < ny - 1; iy++)
          visc_flux(c, cell(c, ix, iy, iz), cell(c, ix, iy + 1, iz), Y_);
    for (int ix = 0; ix < nx; ix++)
      for (int iy = 0; iy < ny; iy++)
        for (int iz = 0; iz < nz - 1; iz++)
          visc_flux(c, cell(c, ix, iy, iz), cell(c, ix, iy, iz + 1), Z_);
    for (int iy = 0; iy < ny; iy++)
      for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++) {
          const long i = cell(c, ix, iy, iz);
          visc_source_step(c, i);
          updateByViscFlux(c, i);
          clearFlux(c, i);
        }
  }
  correctImagCells(c, 1);
  *tau = c->tau;
  free(c->flux);
  free(c->dm);
  free(c->pi0);
  free(c->piH0);
  free(c->Pi0);
  free(c->PiH0);
  return c->err;
}

/* ----------------------------------------------------- test entry points */

void or_transform_pv(const or_eos *eos, const double *Q, int n, double *out) {
  for (int i = 0; i < n; i++) {
    double q[7];
    for (int k = 0; k < 7; k++) q[k] = Q[7 * i + k];
    double *o = out + 8 * i;
    transform_pv(eos, q, &o[0], &o[1], &o[2], &o[3], &o[4], &o[5], &o[6], &o[7]);
  }
}

void or_transport_eval(const or_trc *tr, const double *in, int n, double *out) {
  for (int i = 0; i < n; i++) {
    const double *a = in + 6 * i;
    double *o = out + 4 * i;
    o[0] = tr_etaS(tr, a[0], a[1], a[2], a[3], a[4], a[5]);
    o[1] = tr_zetaS(tr, a[0], a[2], a[4], a[5]);
    tr_getTau(tr, a[0], a[1], a[2], a[3], a[4], a[5], &o[2], &o[3]);
  }
}

/* out[n][6] = p, T, muB, muS, EoS::p, EoS::s (nq = ns = 0) */
void or_eos_full(const or_eos *E, const double *in, int n, double *out) {
  for (int i = 0; i < n; i++) {
    const double *a = in + 4 * i;
    double *o = out + 5 * i;
    if (E->kind == 3) {
      eos3f(E, a[0], a[1], a[2], a[3], &o[1], &o[2], &o[3], &o[4], &o[0]);
    } else if (E->kind == 4) {
      eos_hadron(E, a[0], a[1], a[2], &o[1], &o[2], &o[3], &o[4], &o[0]);
    } else if (E->kind == 5) {
      eos_smash(E, a[0], a[1], a[2], &o[1], &o[2], &o[3], &o[4], &o[0]);
    } else {
      eos_eval5(E, a[0], a[1], &o[1], &o[2], &o[3], &o[4], &o[0]);
    }
  }
}

void or_eos6(const or_eos *eos, const double *e, const double *nb, int n, double *out) {
  for (int i = 0; i < n; i++) {
    double *o = out + 6 * i;
    eos_eval4(eos, e[i], nb[i], &o[1], &o[2], &o[3], &o[0]);
    o[4] = eos_p(eos, e[i], nb[i]);
    o[5] = eos_s(eos, e[i], nb[i], 0., 0.);
  }
}

void or_eos_eval(const or_eos *eos, const double *e, const double *nb, int n,
                 double *out) {
  for (int i = 0; i < n; i++) {
    double T, mub, p;
    eos_eval(eos, e[i], nb[i], &T, &mub, &p);
    out[3 * i] = p;
    out[3 * i + 1] = T;
    out[3 * i + 2] = mub;
  }
}

void or_eos_s(const or_eos *eos, const double *e, const double *nb, int n,
              double *out) {
  for (int i = 0; i < n; i++) out[i] = eos_s(eos, e[i], nb[i], 0., 0.);
}

void or_update_m(const or_grid *g, double *m, double tau, double dt) {
  Ctx cx;
  memset(&cx, 0, sizeof(cx));
  or_state st;
  memset(&st, 0, sizeof(st));
  st.m = m;
  cx.g = g;
  cx.s = &st;
  cx.nx = g->nx;
  cx.ny = g->ny;
  cx.nz = g->nz;
  cx.N = (long)g->nx * g->ny * g->nz;
  cx.dx = (g->xmax - g->xmin) / (g->nx - 1);
  cx.dy = (g->ymax - g->ymin) / (g->ny - 1);
  cx.dz = grid_dz(g);
  cx.dm = (double *)calloc((size_t)(3 * cx.N), sizeof(double));
  updateM(&cx, tau, dt);
  free(cx.dm);
}

/* ------------------------------------------------------------- totals */

/* Fluid::getCMFvariables, src/fld.cpp:50-60: con2prim of Q/tau, then the
 * fluid rapidity Y and the velocities in the fireball rest frame. */
static void cmf_variables(const or_eos *E, const or_state *s, long N, long i,
                          double eta, double tau, double *e, double *nb,
                          double *nq, double *ns, double *vx, double *vy,
                          double *Y) {
  double q[7], p, vz;
  for (int k = 0; k < 7; k++) q[k] = s->Q[(long)k * N + i] / tau;
  transform_pv(E, q, e, &p, nb, nq, ns, vx, vy, &vz);
  *Y = eta + 1. / 2. * log((1. + vz) / (1. - vz));
  *vx = *vx * cosh(*Y - eta) / cosh(*Y);
  *vy = *vy * cosh(*Y - eta) / cosh(*Y);
}

void or_totals(const or_grid *g, const or_eos *E, const or_trc *tr,
               const or_state *s, double tau, double ecrit, double *out) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const long N = (long)nx * ny * nz;
  const double dx = (g->xmax - g->xmin) / (nx - 1);
  const double dy = (g->ymax - g->ymin) / (ny - 1);
  const double dz = grid_dz(g);
  const int visc = tr_isViscous(tr);
  double E_ = 0., Efull = 0., S = 0., Px = 0., vt_num = 0., vt_den = 0.,
         vxvy_num = 0., vxvy_den = 0., pi0x_num = 0., pi0x_den = 0.,
         txxyy_num = 0., txxyy_den = 0., Nb1 = 0., Nb2 = 0.;
  int nCore = 0, nCoreCut = 0;
  const double gmumu[4] = {1., -1., -1., -1.};
  for (int ix = 2; ix < nx - 2; ix++)
    for (int iy = 2; iy < ny - 2; iy++)
      for (int iz = 2; iz < nz - 2; iz++) {
        const long i = ix + (long)nx * iy + (long)nx * ny * iz;
        const double etaz = g->zmin + iz * dz;
        double e, nb, nq, ns, vx, vy, vz, t, mub, p;
        cmf_variables(E, s, N, i, etaz, tau, &e, &nb, &nq, &ns, &vx, &vy, &vz);
        eos_eval(E, e, nb, &t, &mub, &p);
        double sd = eos_s(E, e, nb, nq, ns);
        const double eta = etaz;
        const double cosh_int = (sinh(eta + 0.5 * dz) - sinh(eta - 0.5 * dz)) / dz;
        const double sinh_int = (cosh(eta + 0.5 * dz) - cosh(eta - 0.5 * dz)) / dz;
        E_ += tau * (e + p) / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz)) *
                  (cosh_int - tanh(vz) * sinh_int) -
              tau * p * cosh_int;
        Nb1 += s->Q[(long)NB_ * N + i];
        Nb2 += tau * nb * (cosh_int - tanh(vz) * sinh_int) /
               sqrt(1. - vx * vx - vy * vy - tanh(vz) * tanh(vz));
        Efull += tau * (e + p) / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz)) *
                     (cosh(eta) - tanh(vz) * sinh(eta)) -
                 tau * p * cosh(eta);
        const double pi00 = s->pi[(long)index44(0, 0) * N + i];
        const double pi03 = s->pi[(long)index44(0, 3) * N + i];
        const double pi01 = s->pi[(long)index44(0, 1) * N + i];
        if (visc) Efull += tau * pi00 * cosh(eta) + tau * pi03 * sinh(eta);
        if (e > ecrit) {
          nCore++;
          if (s->vcc[i] < 0.9) nCoreCut++;
        }
        double deltas = 0.;
        if (visc)
          for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
              const double pab = s->pi[(long)index44(a, b) * N + i];
              deltas += pab * pab * gmumu[a] * gmumu[b];
            }
        if (t > 0.02) {
          sd += 1.5 * deltas / ((e + p) * t);
          S += tau * sd * (cosh_int - tanh(vz) * sinh_int) /
               sqrt(1. - vx * vx - vy * vy - tanh(vz) * tanh(vz));
        }
        Px += tau * (e + p) * vx / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz));
        if (iz > nz / 2 - 3 && iz < nz / 2 + 3) {
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
        pi0x_num += e / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz)) * fabs(pi01);
        pi0x_den += e / (1. - vx * vx - vy * vy - tanh(vz) * tanh(vz));
      }
  out[0] = E_ * dx * dy * dz;
  out[1] = Efull * dx * dy * dz;
  out[2] = Nb1 * (dx * dy * dz);
  out[3] = Nb2 * (dx * dy * dz);
  out[4] = S * dx * dy * dz;
  out[5] = Px;
  out[6] = vt_num;
  out[7] = vt_den;
  out[8] = vxvy_num;
  out[9] = vxvy_den;
  out[10] = pi0x_num;
  out[11] = pi0x_den;
  out[12] = txxyy_num;
  out[13] = txxyy_den;
  out[14] = nCore;
  out[15] = nCoreCut;
}

/* expandGrid2x, src/main.cpp:246-271.  The new grid keeps nx, ny, nz and
 * spans twice the transverse range, its bounds taken from the old grid's
 * first and last cell coordinates (Fluid::getX = minx + ix*dx, src/fld.h);
 * each new cell imports every variable of the old cell at
 * 2*(i - n/2) + n/2 (clamped like Fluid::getCell) in x and y and the same iz
 * (Cell::importVars, src/cll.cpp:54-68). */
int or_resize2x(const or_grid *g, const or_state *in, or_grid *gout,
                or_state *out) {
  const double dx = (g->xmax - g->xmin) / (g->nx - 1);
  const double dy = (g->ymax - g->ymin) / (g->ny - 1);
  const double dz = grid_dz(g);
  const double x0 = g->xmin + 0 * dx, x1 = g->xmin + (g->nx - 1) * dx;
  const double y0 = g->ymin + 0 * dy, y1 = g->ymin + (g->ny - 1) * dy;
  if (x0 + x1 > 0.001 || y0 + y1 > 0.001) return 0;
  or_grid ng = *g;
  ng.xmin = 2.0 * x0;
  ng.xmax = 2.0 * x1;
  ng.ymin = 2.0 * y0;
  ng.ymax = 2.0 * y1;
  ng.zmin = g->zmin + 0 * dz;
  ng.zmax = g->zmin + (g->nz - 1) * dz;
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const long N = (long)nx * ny * nz;
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < ny; iy++)
      for (int ix = 0; ix < nx; ix++) {
        int sx = 2 * (ix - nx / 2) + nx / 2, sy = 2 * (iy - ny / 2) + ny / 2;
        sx = sx > 0 ? sx : 0;
        sx = sx < nx ? sx : nx - 1;
        sy = sy > 0 ? sy : 0;
        sy = sy < ny ? sy : ny - 1;
        const long i = ix + (long)nx * (iy + (long)ny * iz);
        const long j = sx + (long)nx * (sy + (long)ny * iz);
        for (int k = 0; k < 7; k++) {
          out->Q[k * N + i] = in->Q[k * N + j];
          out->Qh[k * N + i] = in->Qh[k * N + j];
          out->Qprev[k * N + i] = in->Qprev[k * N + j];
        }
        for (int k = 0; k < 10; k++) {
          out->pi[k * N + i] = in->pi[k * N + j];
          out->piH[k * N + i] = in->piH[k * N + j];
        }
        out->Pi[i] = in->Pi[j];
        out->PiH[i] = in->PiH[j];
        for (int k = 0; k < 3; k++) out->m[k * N + i] = in->m[k * N + j];
        out->vcc[i] = in->vcc[j];
      }
  *gout = ng;
  return 1;
}

/* The driver's substep count, src/main.cpp:405-409: halve the step until
 * it is below tau times the eta cell size of the parameters' grid.  Returns
 * -1 when the count would pass 2^30. */
int or_substeps(double dtau, double tau, double etamin, double etamax, int nz) {
  int n = 1;
  while (dtau / n > 1.0 * tau * (etamax - etamin) / (nz - 1)) {
    if (n >= (1 << 30)) return -1;
    n *= 2;
  }
  return n;
}

/* ===================================================================
 * Freeze-out hypersurface: Cornelius 4D (P. Huovinen and H. Petersen,
 * Eur. Phys. J. A 48 (2012) 171, arXiv:1206.3371) as the reference's
 * cornelius.cpp implements it, restated over flat arrays.
 *
 * Hypercube corner values cube[it*8 + jx*4 + jy*2 + jz] (dimension 0 is
 * time).  The 4-cube splits into 8 3-cubes (constant dimension i at j = 0, 1,
 * Hypercube::split_to_cubes, cornelius.cpp:1733-1774), each 3-cube into 6
 * squares (Cube::split_to_squares, :1436-1482).  A square yields 0-2 line
 * elements (Square::construct_lines / ends_of_edge / find_outside,
 * :1083-1313), a 3-cube joins its lines into polygons (:1484-1578), the
 * 4-cube joins polygons into polyhedra (:1776-1878); each polyhedron is one
 * surface element whose centroid and normal come from its tetrahedra
 * (:761-1000).
 * =================================================================== */
#define CN_MAX_LINES 96
#define CN_MAX_POLY 64
#define CN_MAX_POLY_PER_CUBE 8
#define CN_MAX_ELEM 10
#define CN_EPS 1e-10

typedef struct cn_line {
  double p[2][4]; /* the two end points */
  double o[4];    /* a point outside the surface */
  int start;      /* index of the start point in p (flip_start_end swaps) */
} cn_line;

typedef struct cn_poly {
  int n, cdim;
  int li[12];
  double cen[4];
} cn_poly;

typedef struct cn_work {
  cn_line L[CN_MAX_LINES];
  int nl;
  cn_poly P[CN_MAX_POLY];
  int np;
  int err;
} cn_work;

static const double *ln_start(const cn_line *l) { return l->p[l->start]; }
static const double *ln_end(const cn_line *l) { return l->p[1 - l->start]; }

static double hv(const double *cube, const int b[4]) {
  return cube[b[0] * 8 + b[1] * 4 + b[2] * 2 + b[3]];
}

/* Square::construct_lines (cornelius.cpp:1083-1133) for the square whose
 * constant dimensions are c0, c1 (values v0, v1) and whose corner values
 * are p[a][b] (a along x1, b along x2, x1 < x2).  Appends its lines to w
 * and returns 1 when the square is ambiguous (4 cuts). */
static int cn_square(cn_work *w, const double p[2][2], int c0, int c1, double v0,
                     double v1, int x1, int x2, const double *dx, double E0) {
  int above = 0;
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++)
      if (p[i][j] >= E0) above++;
  if (above == 0 || above == 4) return 0;
  double cuts[4][2], out[2][2];
  int nc = 0, amb = 0;
  /* ends_of_edge, :1147-1221 */
  if ((p[0][0] - E0) * (p[1][0] - E0) < 0) {
    cuts[nc][0] = (p[0][0] - E0) / (p[0][0] - p[1][0]) * dx[x1];
    cuts[nc++][1] = 0;
  } else if (p[0][0] == E0 && p[1][0] < E0) {
    cuts[nc][0] = 1e-9 * dx[x1];
    cuts[nc++][1] = 0;
  } else if (p[1][0] == E0 && p[0][0] < E0) {
    cuts[nc][0] = (1.0 - 1e-9) * dx[x1];
    cuts[nc++][1] = 0;
  }
  if ((p[0][0] - E0) * (p[0][1] - E0) < 0) {
    cuts[nc][0] = 0;
    cuts[nc++][1] = (p[0][0] - E0) / (p[0][0] - p[0][1]) * dx[x2];
  } else if (p[0][0] == E0 && p[0][1] < E0) {
    cuts[nc][0] = 0;
    cuts[nc++][1] = 1e-9 * dx[x2];
  } else if (p[0][1] == E0 && p[0][0] < E0) {
    cuts[nc][0] = 0;
    cuts[nc++][1] = (1.0 - 1e-9) * dx[x2];
  }
  if ((p[1][0] - E0) * (p[1][1] - E0) < 0) {
    cuts[nc][0] = dx[x1];
    cuts[nc++][1] = (p[1][0] - E0) / (p[1][0] - p[1][1]) * dx[x2];
  } else if (p[1][0] == E0 && p[1][1] < E0) {
    cuts[nc][0] = dx[x1];
    cuts[nc++][1] = 1e-9 * dx[x2];
  } else if (p[1][1] == E0 && p[1][0] < E0) {
    cuts[nc][0] = dx[x1];
    cuts[nc++][1] = (1.0 - 1e-9) * dx[x2];
  }
  if ((p[0][1] - E0) * (p[1][1] - E0) < 0) {
    cuts[nc][0] = (p[0][1] - E0) / (p[0][1] - p[1][1]) * dx[x1];
    cuts[nc++][1] = dx[x2];
  } else if (p[0][1] == E0 && p[1][1] < E0) {
    cuts[nc][0] = 1e-9 * dx[x1];
    cuts[nc++][1] = dx[x2];
  } else if (p[1][1] == E0 && p[0][1] < E0) {
    cuts[nc][0] = (1.0 - 1e-9) * dx[x1];
    cuts[nc++][1] = dx[x2];
  }
  if (nc != 0 && nc != 2 && nc != 4) { /* the reference exits */
    w->err |= 1;
    return 0;
  }
  if (nc == 0) return 0;
  /* find_outside, :1223-1298 */
  if (nc == 4) {
    amb = 1;
    double Emid = 0;
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) Emid += 0.25 * p[i][j];
    if ((p[0][0] < E0 && Emid < E0) || (p[0][0] > E0 && Emid > E0)) {
      for (int i = 0; i < 2; i++) {
        const double t = cuts[1][i];
        cuts[1][i] = cuts[2][i];
        cuts[2][i] = t;
      }
    }
    if ((Emid - E0) < 0) {
      out[0][0] = out[1][0] = 0.5 * dx[x1];
      out[0][1] = out[1][1] = 0.5 * dx[x2];
    } else if ((p[0][0] - E0) < 0) {
      out[0][0] = 0;
      out[0][1] = 0;
      out[1][0] = dx[x1];
      out[1][1] = dx[x2];
    } else {
      out[0][0] = dx[x1];
      out[0][1] = 0;
      out[1][0] = 0;
      out[1][1] = dx[x2];
    }
  } else {
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) out[i][j] = 0;
    int nout = 0;
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++)
        if (p[i][j] < E0) {
          out[0][0] += i * dx[x1];
          out[0][1] += j * dx[x2];
          nout++;
        }
    if (nout > 0)
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) out[i][j] = out[i][j] / (double)nout;
  }
  for (int k = 0; k < nc / 2; k++) {
    if (w->nl >= CN_MAX_LINES) {
      w->err |= 2;
      return amb;
    }
    cn_line *l = &w->L[w->nl++];
    for (int e = 0; e < 2; e++) {
      l->p[e][x1] = cuts[2 * k + e][0];
      l->p[e][x2] = cuts[2 * k + e][1];
      l->p[e][c0] = v0;
      l->p[e][c1] = v1;
    }
    l->o[x1] = out[k][0];
    l->o[x2] = out[k][1];
    l->o[c0] = v0;
    l->o[c1] = v1;
    l->start = 0;
  }
  return amb;
}

/* Polygon::add_line (cornelius.cpp:404-438) */
static int cn_add_line(cn_work *w, cn_poly *pg, int li, int donotcheck) {
  if (donotcheck || pg->n == 0) {
    pg->li[pg->n++] = li;
    return 1;
  }
  cn_line *l = &w->L[li];
  const double *p1 = ln_start(l), *p2 = ln_end(l), *p3 = ln_end(&w->L[pg->li[pg->n - 1]]);
  double d1 = 0, d2 = 0;
  for (int j = 0; j < 4; j++) {
    d1 += fabs(p1[j] - p3[j]);
    d2 += fabs(p2[j] - p3[j]);
  }
  if (d1 < CN_EPS || d2 < CN_EPS) {
    if (d2 < CN_EPS) l->start = 1 - l->start;
    pg->li[pg->n++] = li;
    return 1;
  }
  return 0;
}

/* Cube::construct_polygons (cornelius.cpp:1484-1578) for the 3-cube with
 * constant dimension ci at corner bit jc.  Returns its line count. */
static int cn_cube(cn_work *w, const double *cube, int ci, int jc, const double *dx,
                   double E0, int *cube_amb) {
  const int l0 = w->nl, p0 = w->np;
  const double cv = jc * dx[ci];
  int namb = 0;
  for (int i = 0; i < 4; i++) {
    if (i == ci) continue;
    int x1 = -1, x2 = -1;
    for (int d = 0; d < 4; d++)
      if (d != ci && d != i) {
        if (x1 < 0)
          x1 = d;
        else
          x2 = d;
      }
    for (int j = 0; j < 2; j++) {
      double sq[2][2];
      for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) {
          int bits[4];
          bits[ci] = jc;
          bits[i] = j;
          bits[x1] = a;
          bits[x2] = b;
          sq[a][b] = hv(cube, bits);
        }
      namb += cn_square(w, sq, ci, i, cv, j * dx[i], x1, x2, dx, E0);
    }
  }
  const int nl = w->nl - l0;
  *cube_amb = 0;
  if (nl == 0) return 0;
  /* Cube::check_ambiguous, :1580-1595 */
  int amb = namb;
  if (amb == 0 && nl == 6) amb = 1;
  *cube_amb = amb;
  if (amb > 0) {
    int not_used[CN_MAX_LINES];
    for (int i = 0; i < nl; i++) not_used[i] = 1;
    int used = 0;
    do {
      /* the reference exits (too few lines) or overflows its polygon array */
      if (nl - used < 3 || w->np >= CN_MAX_POLY || w->np - p0 >= CN_MAX_POLY_PER_CUBE) {
        w->err |= 4;
        return nl;
      }
      cn_poly *pg = &w->P[w->np];
      pg->n = 0;
      pg->cdim = ci;
      for (int i = 0; i < nl; i++) {
        if (not_used[i]) {
          if (cn_add_line(w, pg, l0 + i, 0)) {
            not_used[i] = 0;
            used++;
            i = 0;
          }
        }
      }
      w->np++;
    } while (used < nl);
  } else {
    if (w->np >= CN_MAX_POLY) {
      w->err |= 4;
      return nl;
    }
    cn_poly *pg = &w->P[w->np];
    pg->n = 0;
    pg->cdim = ci;
    for (int i = 0; i < nl; i++) cn_add_line(w, pg, l0 + i, 1);
    w->np++;
  }
  return nl;
}

/* Polygon::calculate_centroid (cornelius.cpp:440-516) */
static void cn_poly_centroid(const cn_work *w, cn_poly *pg) {
  int x[3], k = 0;
  for (int d = 0; d < 4; d++)
    if (d != pg->cdim) x[k++] = d;
  const int x1 = x[0], x2 = x[1], x3 = x[2];
  double mean[4] = {0, 0, 0, 0};
  for (int i = 0; i < pg->n; i++) {
    const cn_line *l = &w->L[pg->li[i]];
    const double *p1 = ln_start(l), *p2 = ln_end(l);
    for (int j = 0; j < 4; j++) mean[j] += p1[j] + p2[j];
  }
  for (int j = 0; j < 4; j++) mean[j] = mean[j] / (double)(2.0 * pg->n);
  if (pg->n == 3) {
    for (int j = 0; j < 4; j++) pg->cen[j] = mean[j];
    return;
  }
  double up[4] = {0, 0, 0, 0}, down = 0, a[4], b[4], cm[4];
  for (int i = 0; i < pg->n; i++) {
    const cn_line *l = &w->L[pg->li[i]];
    const double *p1 = ln_start(l), *p2 = ln_end(l);
    for (int j = 0; j < 4; j++) cm[j] = (p1[j] + p2[j] + mean[j]) / 3.0;
    for (int j = 0; j < 4; j++) {
      a[j] = p1[j] - mean[j];
      b[j] = p2[j] - mean[j];
    }
    const double c1 = a[x2] * b[x3] - a[x3] * b[x2];
    const double c2 = a[x1] * b[x3] - a[x3] * b[x1];
    const double c3 = a[x2] * b[x1] - a[x1] * b[x2];
    const double A = 0.5 * sqrt(c1 * c1 + c2 * c2 + c3 * c3);
    for (int j = 0; j < 4; j++) up[j] += cm[j] * A;
    down += A;
  }
  for (int j = 0; j < 4; j++) pg->cen[j] = up[j] / down;
}

/* Polyhedron::tetravolume (cornelius.cpp:771-788) */
static void cn_tetra(const double *a, const double *b, const double *c, double *n) {
  const double bc01 = b[0] * c[1] - b[1] * c[0];
  const double bc02 = b[0] * c[2] - b[2] * c[0];
  const double bc03 = b[0] * c[3] - b[3] * c[0];
  const double bc12 = b[1] * c[2] - b[2] * c[1];
  const double bc13 = b[1] * c[3] - b[3] * c[1];
  const double bc23 = b[2] * c[3] - b[3] * c[2];
  n[0] = 1.0 / 6.0 * (a[1] * bc23 - a[2] * bc13 + a[3] * bc12);
  n[1] = -1.0 / 6.0 * (a[0] * bc23 - a[2] * bc03 + a[3] * bc02);
  n[2] = 1.0 / 6.0 * (a[0] * bc13 - a[1] * bc03 + a[3] * bc01);
  n[3] = -1.0 / 6.0 * (a[0] * bc12 - a[1] * bc02 + a[2] * bc01);
}

/* Polyhedron::lines_equal (cornelius.cpp:749-765) */
static int cn_lines_equal(const cn_line *l1, const cn_line *l2) {
  const double *p11 = ln_start(l1), *p12 = ln_end(l1), *p21 = ln_start(l2);
  double d1 = 0, d2 = 0;
  for (int i = 0; i < 4; i++) {
    d1 += fabs(p11[i] - p21[i]);
    d2 += fabs(p12[i] - p21[i]);
    if (d1 > CN_EPS && d2 > CN_EPS) return 0;
  }
  return 1;
}

/* Cornelius::find_surface_4d (cornelius.cpp:2247-2285) with Hypercube
 * construct_polyhedrons / check_ambiguous (:1776-1878): returns the number
 * of elements (centroid, normal relative to the cube's low corner), or -1
 * when the reference would have stopped (exit or overflow). */
int or_cornelius4d(const double cube[16], const double dx[4], double E0, double cent[][4],
                   double norm[][4]) {
  int above = 0;
  for (int k = 0; k < 16; k++)
    if (cube[k] >= E0) above++;
  if (above == 0 || above == 16) return 0;
  static cn_work w; /* single-threaded oracle */
  w.nl = w.np = w.err = 0;
  int namb = 0, nlines = 0;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 2; j++) {
      int ca;
      nlines += cn_cube(&w, cube, i, j, dx, E0, &ca);
      if (ca) namb++;
    }
  if (w.err) return -1;
  int amb = namb;
  if (amb == 0) {
    int pts = 0;
    for (int k = 0; k < 16; k++)
      if (cube[k] < E0) pts++;
    if (pts > 8) pts = 16 - pts;
    if (nlines == 24 && pts == 2) amb++;
  }
  int ph[CN_MAX_ELEM][CN_MAX_POLY], nph[CN_MAX_ELEM], nel = 0;
  if (amb > 0) {
    int not_used[CN_MAX_POLY], used = 0;
    for (int i = 0; i < w.np; i++) not_used[i] = 1;
    do {
      if (nel >= CN_MAX_ELEM) return -1;
      nph[nel] = 0;
      for (int i = 0; i < w.np; i++) {
        if (!not_used[i]) continue;
        int add = 0;
        if (nph[nel] == 0) {
          add = 1;
        } else {
          const cn_poly *p = &w.P[i];
          for (int q = 0; q < nph[nel] && !add; q++) {
            const cn_poly *pq = &w.P[ph[nel][q]];
            for (int j = 0; j < p->n && !add; j++)
              for (int k = 0; k < pq->n && !add; k++)
                if (cn_lines_equal(&w.L[p->li[j]], &w.L[pq->li[k]])) add = 1;
          }
        }
        if (add) {
          ph[nel][nph[nel]++] = i;
          not_used[i] = 0;
          used++;
          i = 0;
        }
      }
      nel++;
    } while (used < w.np);
  } else {
    nph[0] = 0;
    for (int i = 0; i < w.np; i++) ph[0][nph[0]++] = i;
    nel = 1;
  }
  for (int i = 0; i < w.np; i++) cn_poly_centroid(&w, &w.P[i]);
  for (int e = 0; e < nel; e++) {
    /* Polyhedron::calculate_centroid, :790-870 */
    int ntet = 0;
    double mean[4] = {0, 0, 0, 0};
    for (int q = 0; q < nph[e]; q++) {
      const cn_poly *pg = &w.P[ph[e][q]];
      ntet += pg->n;
      for (int j = 0; j < pg->n; j++) {
        const cn_line *l = &w.L[pg->li[j]];
        const double *p1 = ln_start(l), *p2 = ln_end(l);
        for (int k = 0; k < 4; k++) mean[k] += p1[k] + p2[k];
      }
    }
    for (int k = 0; k < 4; k++) mean[k] = mean[k] / (double)(2.0 * ntet);
    double up[4] = {0, 0, 0, 0}, down = 0, a[4], b[4], c[4], n[4], cm[4];
    for (int q = 0; q < nph[e]; q++) {
      const cn_poly *pg = &w.P[ph[e][q]];
      for (int j = 0; j < pg->n; j++) {
        const cn_line *l = &w.L[pg->li[j]];
        const double *p1 = ln_start(l), *p2 = ln_end(l);
        for (int k = 0; k < 4; k++) cm[k] = (p1[k] + p2[k] + pg->cen[k] + mean[k]) / 4.0;
        for (int k = 0; k < 4; k++) {
          a[k] = p1[k] - mean[k];
          b[k] = p2[k] - mean[k];
          c[k] = pg->cen[k] - mean[k];
        }
        cn_tetra(a, b, c, n);
        double V = 0;
        for (int k = 0; k < 4; k++) V += n[k] * n[k];
        V = sqrt(V);
        for (int k = 0; k < 4; k++) up[k] += cm[k] * V;
        down += V;
      }
    }
    double *C = cent[e];
    for (int k = 0; k < 4; k++) C[k] = up[k] / down;
    /* Polyhedron::calculate_normal, :872-935 */
    double *Nn = norm[e];
    for (int k = 0; k < 4; k++) Nn[k] = 0;
    for (int q = 0; q < nph[e]; q++) {
      const cn_poly *pg = &w.P[ph[e][q]];
      for (int j = 0; j < pg->n; j++) {
        const cn_line *l = &w.L[pg->li[j]];
        const double *p1 = ln_start(l), *p2 = ln_end(l);
        for (int k = 0; k < 4; k++) {
          a[k] = p1[k] - C[k];
          b[k] = p2[k] - C[k];
          c[k] = pg->cen[k] - C[k];
        }
        cn_tetra(a, b, c, n);
        double dot = 0;
        for (int k = 0; k < 4; k++) dot += (l->o[k] - C[k]) * n[k];
        if (dot < 0)
          for (int k = 0; k < 4; k++) n[k] = -n[k];
        for (int k = 0; k < 4; k++) Nn[k] += n[k];
      }
    }
  }
  return nel;
}

/* Cartesian components of pi^{mu nu} at space-time rapidity eta (the OUTPI
 * block of src/fld.cpp:766-790 and :1028-1053), index44 order. */
static void pi_to_cartesian(double ch, double sh, const double *piC, double *pc) {
  pc[0] = ch * ch * piC[0] + 2. * ch * sh * piC[6] + sh * sh * piC[9];
  pc[1] = ch * piC[1] + sh * piC[7];
  pc[3] = ch * piC[3] + sh * piC[8];
  pc[6] = ch * sh * (piC[0] + piC[9]) + (ch * ch + sh * sh) * piC[6];
  pc[2] = piC[2];
  pc[4] = piC[4];
  pc[7] = sh * piC[1] + ch * piC[7];
  pc[5] = piC[5];
  pc[8] = sh * piC[3] + ch * piC[8];
  pc[9] = sh * sh * piC[0] + ch * ch * piC[9] + 2. * sh * ch * piC[6];
}

/* transformToLab, src/fld.cpp:508-513 */
static void to_lab(double eta, double *vx, double *vy, double *vz) {
  const double Y = eta + 1. / 2. * log((1. + *vz) / (1. - *vz));
  *vx = *vx * cosh(Y - eta) / cosh(Y);
  *vy = *vy * cosh(Y - eta) / cosh(Y);
  *vz = tanh(Y);
}

/* The freeze-out part of Fluid::outputSurface (src/fld.cpp:544-842): for
 * every interior cube [ix, ix+1] x [iy, iy+1] x [iz, iz+1] x [tau - dt,
 * tau] (ix, iy, iz in [2, n-2), iz fastest) the energy densities at the
 * 16 corners (getPrimVar of Q at tau, getPrimVarPrev of Qprev at tau - dt,
 * dt = the Fluid's construction-time step) go to Cornelius; each element
 * gets the interpolated state and one record of OR_SURF_REC doubles:
 * position (4), dSigma_mu (4, from the normal of the cube's FIRST element
 * for every element, as the reference does), u^mu (4), T, muB, muQ, muS,
 * pi^{mu nu} in Cartesian components (10, index44 order), Pi, e, nb.
 * acc[OR_SURF_ACC] += nsusp, EtotSurf, nbSurf, vEff increments and the
 * count of elements with T > 0.4 or |muB| > 0.85.  Returns the number of
 * elements (records beyond cap are counted but not written), or -1 when
 * Cornelius would have stopped the reference. */
static long surface_impl(const or_grid *g, const or_eos *E, const or_state *s, double tau,
                         double dtf, double ecrit, double *rec, long cap, double *acc,
                         double *beta) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const long N = (long)nx * ny * nz;
  const double dx = (g->xmax - g->xmin) / (nx - 1);
  const double dy = (g->ymax - g->ymin) / (ny - 1);
  const double dz = grid_dz(g);
  const double arrayDx[4] = {dtf, dx, dy, dz};
  long nel = 0;
  for (int ix = 2; ix < nx - 2; ix++)
    for (int iy = 2; iy < ny - 2; iy++)
      for (int iz = 2; iz < nz - 2; iz++) {
        double cube[16], QCube[2][8][7], piS[8][10], PiS[8], dbS[8][16];
        for (int jx = 0; jx < 2; jx++)
          for (int jy = 0; jy < 2; jy++)
            for (int jz = 0; jz < 2; jz++) {
              const int c = jx * 4 + jy * 2 + jz;
              const long i = (ix + jx) + (long)nx * (iy + jy) + (long)nx * ny * (iz + jz);
              double q[7], e, p, nb, nq, ns, vx, vy, vz;
              for (int k = 0; k < 7; k++) q[k] = s->Q[(long)k * N + i] / tau;
              transform_pv(E, q, &e, &p, &nb, &nq, &ns, &vx, &vy, &vz);
              cube[8 + c] = e;
              for (int k = 0; k < 7; k++) q[k] = s->Qprev[(long)k * N + i] / (tau - dtf);
              transform_pv(E, q, &e, &p, &nb, &nq, &ns, &vx, &vy, &vz);
              cube[c] = e;
              for (int k = 0; k < 7; k++) {
                QCube[1][c][k] = s->Q[(long)k * N + i];
                QCube[0][c][k] = s->Qprev[(long)k * N + i];
              }
              for (int k = 0; k < 10; k++) piS[c][k] = s->pi[(long)k * N + i];
              PiS[c] = s->Pi[i];
              if (beta)
                for (int k = 0; k < 16; k++) dbS[c][k] = s->dbeta[(long)k * N + i];
            }
        double cen[CN_MAX_ELEM][4], nrm[CN_MAX_ELEM][4];
        const int ne = or_cornelius4d(cube, arrayDx, ecrit, cen, nrm);
        if (ne < 0) return -1;
        for (int el = 0; el < ne; el++) {
          const double *C = cen[el];
          double QC[7] = {0., 0., 0., 0., 0., 0., 0.}, piC[10], PiC = 0.;
          for (int k = 0; k < 10; k++) piC[k] = 0.;
          const double wT[2] = {1. - C[0] / dtf, C[0] / dtf};
          const double wX[2] = {1. - C[1] / dx, C[1] / dx};
          const double wY[2] = {1. - C[2] / dy, C[2] / dy};
          const double wZ[2] = {1. - C[3] / dz, C[3] / dz};
          for (int jt = 0; jt < 2; jt++)
            for (int jx = 0; jx < 2; jx++)
              for (int jy = 0; jy < 2; jy++)
                for (int jz = 0; jz < 2; jz++)
                  for (int k = 0; k < 7; k++)
                    QC[k] += QCube[jt][jx * 4 + jy * 2 + jz][k] * wT[jt] * wX[jx] * wY[jy] * wZ[jz];
          for (int k = 0; k < 7; k++) QC[k] = QC[k] / (tau + C[0]);
          double eC, pC, nbC, nqC, nsC = 0.0, vxC, vyC, vzC, TC, mubC, musC;
          transform_pv(E, QC, &eC, &pC, &nbC, &nqC, &nsC, &vxC, &vyC, &vzC);
          double muqC;
          eos_eval5(E, eC, nbC, &TC, &mubC, &muqC, &musC, &pC);
          if (TC > 0.4 || fabs(mubC) > 0.85) acc[4] += 1.;
          if (eC > ecrit * 2.0 || eC < ecrit * 0.5) acc[0] += 1.;
          double dbI[16];
          for (int k = 0; k < 16; k++) dbI[k] = 0.0;
          for (int jx = 0; jx < 2; jx++)
            for (int jy = 0; jy < 2; jy++)
              for (int jz = 0; jz < 2; jz++) {
                const int c = jx * 4 + jy * 2 + jz;
                for (int k = 0; k < 10; k++) piC[k] += piS[c][k] * wX[jx] * wY[jy] * wZ[jz];
                PiC += PiS[c] * wX[jx] * wY[jy] * wZ[jz];
                if (beta) /* src/fld.cpp:716-727 */
                  for (int k = 0; k < 16; k++) dbI[k] += dbS[c][k] * wX[jx] * wY[jy] * wZ[jz];
              }
          double v2C = vxC * vxC + vyC * vyC + vzC * vzC;
          if (v2C > 1.) {
            vxC *= sqrt(0.99 / v2C);
            vyC *= sqrt(0.99 / v2C);
            vzC *= sqrt(0.99 / v2C);
            v2C = 0.99;
          }
          const double etaC = (g->zmin + iz * dz) + C[3];
          to_lab(etaC, &vxC, &vyC, &vzC);
          const double gammaC = 1. / sqrt(1. - vxC * vxC - vyC * vyC - vzC * vzC);
          const double uC[4] = {gammaC, gammaC * vxC, gammaC * vyC, gammaC * vzC};
          const double tauC = tau + C[0];
          const double ch = cosh(etaC), sh = sinh(etaC);
          const double *n0 = nrm[0];
          double ds[4];
          ds[0] = tauC * (ch * n0[0] - sh / tauC * n0[3]);
          ds[3] = tauC * (-sh * n0[0] + ch / tauC * n0[3]);
          ds[1] = tauC * n0[1];
          ds[2] = tauC * n0[2];
          double dVEff = 0.0;
          for (int k = 0; k < 4; k++) dVEff += ds[k] * uC[k];
          double pc[10];
          pc[0] = ch * ch * piC[0] + 2. * ch * sh * piC[6] + sh * sh * piC[9];
          pc[1] = ch * piC[1] + sh * piC[7];
          pc[3] = ch * piC[3] + sh * piC[8];
          pc[6] = ch * sh * (piC[0] + piC[9]) + (ch * ch + sh * sh) * piC[6];
          pc[2] = piC[2];
          pc[4] = piC[4];
          pc[7] = sh * piC[1] + ch * piC[7];
          pc[5] = piC[5];
          pc[8] = sh * piC[3] + ch * piC[8];
          pc[9] = sh * sh * piC[0] + ch * ch * piC[9] + 2. * sh * ch * piC[6];
          const int i0k[4] = {0, 1, 3, 6}; /* index44(0, k) */
          double dEsurfVisc = 0.;
          for (int k = 0; k < 4; k++) dEsurfVisc += pc[i0k[k]] * ds[k];
          acc[1] += (eC + pC) * uC[0] * dVEff - pC * ds[0] + dEsurfVisc;
          acc[2] += nbC * dVEff;
          acc[3] += dVEff;
          if (nel < cap) {
            double *r = rec + nel * OR_SURF_REC;
            r[0] = tau + C[0];
            r[1] = (g->xmin + ix * dx) + C[1];
            r[2] = (g->ymin + iy * dy) + C[2];
            r[3] = (g->zmin + iz * dz) + C[3];
            for (int k = 0; k < 4; k++) {
              r[4 + k] = ds[k];
              r[8 + k] = uC[k];
            }
            r[12] = TC;
            r[13] = mubC;
            r[14] = muqC;
            r[15] = musC;
            for (int k = 0; k < 10; k++) r[16 + k] = pc[k];
            r[26] = PiC;
            r[27] = eC;
            r[28] = nbC;
            if (beta) {
              /* d_i beta_j in Cartesian components: J_ik J_jl dbeta_kl g_ll
               * with the Milne-to-Cartesian Jacobian, src/fld.cpp:798-831 */
              const double J[4][4] = {
                  {ch, 0., 0., -sh}, {0., 1., 0., 0.}, {0., 0., 1., 0.}, {-sh, 0., 0., ch}};
              const double gl[4] = {1., -1., -1., -1.};
              double *b = beta + nel * 16;
              for (int a = 0; a < 4; a++)
                for (int bb = 0; bb < 4; bb++) {
                  double v = 0.0;
                  for (int k = 0; k < 4; k++)
                    for (int l = 0; l < 4; l++) v += J[a][k] * J[bb][l] * dbI[4 * k + l] * gl[l];
                  b[4 * a + bb] = v;
                }
            }
          }
          nel++;
        }
      }
  return nel;
}

long or_surface(const or_grid *g, const or_eos *E, const or_state *s, double tau,
                double dtf, double ecrit, double *rec, long cap, double *acc) {
  return surface_impl(g, E, s, tau, dtf, ecrit, rec, cap, acc, NULL);
}

long or_surface_beta(const or_grid *g, const or_eos *E, const or_state *s, double tau,
                     double dtf, double ecrit, double *rec, long cap, double *acc,
                     double *beta) {
  if (!s->dbeta) return -2;
  return surface_impl(g, E, s, tau, dtf, ecrit, rec, cap, acc, beta);
}

/* Fluid::outputCorona, src/fld.cpp:876-1089 (the element part; the totals
 * it prints are or_totals').  Loop order ix, iy, iz (iz fastest) over
 * [2, n-2). */
long or_corona(const or_grid *g, const or_eos *E, const or_state *s, double tau,
               double ecrit, double *rec, long cap, double *acc) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const long N = (long)nx * ny * nz;
  const double dx = (g->xmax - g->xmin) / (nx - 1);
  const double dy = (g->ymax - g->ymin) / (ny - 1);
  const double dz = grid_dz(g);
  long nel = 0;
  for (int ix = 2; ix < nx - 2; ix++)
    for (int iy = 2; iy < ny - 2; iy++)
      for (int iz = 2; iz < nz - 2; iz++) {
        int isCorona = 1;
        double QCube[8][7], piS[8][10], PiS[8];
        for (int jx = 0; jx < 2; jx++)
          for (int jy = 0; jy < 2; jy++)
            for (int jz = 0; jz < 2; jz++) {
              const int c = jx * 4 + jy * 2 + jz;
              const long i = (ix + jx) + (long)nx * (iy + jy) + (long)nx * ny * (iz + jz);
              double q[7], e, p, nb, nq, ns, vx, vy, vz;
              /* Cell::getPrimVar, src/cll.cpp:90-95 */
              for (int k = 0; k < 7; k++) q[k] = s->Q[(long)k * N + i] / tau;
              transform_pv(E, q, &e, &p, &nb, &nq, &ns, &vx, &vy, &vz);
              for (int k = 0; k < 7; k++) QCube[c][k] = s->Q[(long)k * N + i];
              if (e > ecrit) isCorona = 0;
              for (int k = 0; k < 10; k++) piS[c][k] = s->pi[(long)k * N + i];
              PiS[c] = s->Pi[i];
            }
        double QC[7] = {0., 0., 0., 0., 0., 0., 0.};
        for (int c = 0; c < 8; c++)
          for (int k = 0; k < 7; k++) QC[k] += QCube[c][k] * 0.125;
        for (int k = 0; k < 7; k++) QC[k] = QC[k] / tau;
        double eC, pC, nbC, nqC, nsC = 0.0, vxC, vyC, vzC, TC, mubC;
        transform_pv(E, QC, &eC, &pC, &nbC, &nqC, &nsC, &vxC, &vyC, &vzC);
        const int isTail = !(eC >= 0.01);
        if (!isCorona || isTail) continue;
        double musC;
        double muqC;
        eos_eval5(E, eC, nbC, &TC, &mubC, &muqC, &musC, &pC);
        if (TC > 0.4 || fabs(mubC) > 0.99) acc[4] += 1.;
        double piC[10], PiC = 0.;
        for (int k = 0; k < 10; k++) piC[k] = 0.;
        for (int c = 0; c < 8; c++) {
          for (int k = 0; k < 10; k++) piC[k] += piS[c][k] * 0.125;
          PiC += PiS[c] * 0.125;
        }
        double v2C = vxC * vxC + vyC * vyC + vzC * vzC;
        if (v2C > 1.) {
          vxC *= sqrt(0.99 / v2C);
          vyC *= sqrt(0.99 / v2C);
          vzC *= sqrt(0.99 / v2C);
          v2C = 0.99;
        }
        const double etaC = (g->zmin + iz * dz) + 0.5 * dz;
        to_lab(etaC, &vxC, &vyC, &vzC);
        const double gammaC = 1. / sqrt(1. - vxC * vxC - vyC * vyC - vzC * vzC);
        const double uC[4] = {gammaC, gammaC * vxC, gammaC * vyC, gammaC * vzC};
        const double ch = cosh(etaC), sh = sinh(etaC);
        double ds[4];
        ds[0] = tau * (ch * dx * dy * dz);
        ds[3] = tau * (-sh * dx * dy * dz);
        ds[1] = 0.0;
        ds[2] = 0.0;
        double dVEff = 0.0;
        for (int k = 0; k < 4; k++) dVEff += ds[k] * uC[k];
        double pc[10];
        pi_to_cartesian(ch, sh, piC, pc);
        const int i0k[4] = {0, 1, 3, 6}; /* index44(0, k) */
        double dEsurfVisc = 0.;
        for (int k = 0; k < 4; k++) dEsurfVisc += pc[i0k[k]] * ds[k];
        acc[1] += (eC + pC) * uC[0] * dVEff - pC * ds[0] + dEsurfVisc;
        acc[2] += nbC * dVEff;
        acc[3] += dVEff;
        if (nel < cap) {
          double *r = rec + nel * OR_SURF_REC;
          r[0] = tau;
          r[1] = (g->xmin + ix * dx) + 0.5 * dx;
          r[2] = (g->ymin + iy * dy) + 0.5 * dy;
          r[3] = (g->zmin + iz * dz) + 0.5 * dz;
          for (int k = 0; k < 4; k++) {
            r[4 + k] = ds[k];
            r[8 + k] = uC[k];
          }
          r[12] = TC;
          r[13] = mubC;
          r[14] = muqC;
          r[15] = musC;
          for (int k = 0; k < 10; k++) r[16 + k] = pc[k];
          r[26] = PiC;
          r[27] = eC;
          r[28] = nbC;
        }
        nel++;
      }
  return nel;
}
