/*
 * vh_oracle_ic.c -- CPU oracle for the reference's initial-state modules.
 *
 * TEST INFRASTRUCTURE ONLY.  A plain-C, single-threaded restatement of the
 * IC classes the reference driver selects by icModel (src/main.cpp:324-366)
 * and of the s95p entropy-to-energy inversion they share (src/s95p.cpp):
 *   or_ic_glissando  IcGlissando (src/icGlissando.cpp), icModel 5
 *   or_ic_trento     IcTrento (src/icTrento.cpp), icModel 7
 *   or_ic_gubser     ICGubser (src/icGubser.cpp), icModel 4
 *   or_ic_table      IC + s95p::loadSongIC / getSongEps (src/ic.cpp,
 *                    src/s95p.cpp:43-88), icModel 2
 *   or_ic_urqmd      IcPartUrqmd (src/icPartUrqmd.cpp), icModel 3
 * over the structure-of-arrays state of vh_oracle.h.  It checks the CUDA
 * builders (vh_init_glissando, vh_init_trento, vh_init_gubser,
 * vh_init_table); the product never links, loads or calls it.
 *
 * Parity pin: every function here is compared with the reference's own
 * classes compiled unmodified into oracle/_ref (ref_ic, ref_s95p_e in
 * oracle/ref_harness.cpp) by tests/test_oracle_ic.py.
 *
 * crmath = 0 evaluates exp and pow with the C library, as the reference
 * does; crmath = 1 evaluates the per-cell and per-source ones (the
 * smearing's exp, the s95p inversion, the Gubser profile) with the
 * correctly rounded or_exp_cr / or_pow_cr of the CUDA path (and pow(x, 2) as
 * x * x), and the per-axis factors (the rapidity profiles, the table IC's
 * eta factor, cosh, tanh, sinh) with the C library, as the CUDA path's host
 * side does; so the two arms separate the library's rare misrounded last
 * bits from everything else.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vh_oracle.h"

static const double OR_C_PI = 3.14159265358979312; /* src/inc.h:18 */

static double xexp(double x, int cr) { return cr ? or_exp_cr(x) : exp(x); }
static double xpow(double x, double y, int cr) { return cr ? or_pow_cr(x, y) : pow(x, y); }
static double xsq(double x, int cr) { return cr ? x * x : pow(x, 2); }

/* s95p::s95p_s, src/s95p.cpp:14-32: the s95p-PCE parametrisation of the
 * entropy density (fm^-3) against e (GeV/fm^3) */
double or_s95p_s(double e, int cr) {
  double val;
  if (e < 0.1270769021427449)
    val = 12.2304 * xpow(e, 1.16849, cr);
  else if (e < 0.4467079524674040)
    val = 11.9279 * xpow(e, 1.15635, cr);
  else if (e < 1.9402832534193788)
    val = 0.0580578 + 11.833 * xpow(e, 1.16187, cr);
  else if (e < 3.7292474570977285)
    val = 18.202 * e - 62.021814 - 4.85479 * xexp(-2.72407e-11 * xpow(e, 4.54886, cr), cr) +
          65.1272 * xpow(e, -0.128012, cr) * xexp(-0.00369624 * xpow(e, 1.18735, cr), cr) -
          4.75253 * xpow(e, -1.18423, cr);
  else
    val = 18.202 * e - 63.0218 - 4.85479 * xexp(-2.72407e-11 * xpow(e, 4.54886, cr), cr) +
          65.1272 * xpow(e, -0.128012, cr) * xexp(-0.00369624 * xpow(e, 1.18735, cr), cr);
  return xpow(val, 3. / 4., cr);
}

/* s95p::s95p_e, src/s95p.cpp:34-41: Newton's method on s95p_s from
 * e = s^(4/3) / 18.2, until one step moves e by at most 1e-10 */
double or_s95p_e(double s, int cr) {
  double e = xpow(s, 4. / 3., cr) / 18.2, e0;
  do {
    e0 = e;
    e = e0 - (or_s95p_s(e0, cr) - s) / (6.608681233 * xpow(e0, -0.25, cr));
  } while (fabs(e - e0) > 1e-10);
  return e;
}

/* Fluid's cell sizes and coordinates (src/fld.cpp:77-79, src/fld.h:62-64) */
static double gdx(const or_grid *g) { return (g->xmax - g->xmin) / (g->nx - 1); }
static double gdy(const or_grid *g) { return (g->ymax - g->ymin) / (g->ny - 1); }
static double gdz(const or_grid *g) {
  return g->dz > 0. ? g->dz : (g->zmax - g->zmin) / (g->nz - 1);
}

/* EoS::p at (e, nb, nq, ns) through or_eos_full */
static double eos_p4(const or_eos *E, double e, double nb, double nq, double ns) {
  const double in[4] = {e, nb, nq, ns};
  double out[5];
  or_eos_full(E, in, 1, out);
  return out[0];
}

/* Cell::setPrimVar, src/cll.cpp:222-241 */
static void set_prim_var(const or_eos *E, double *Q, long N, long i, double tau, double e,
                         double nb, double nq, double ns, double vx, double vy, double vz) {
  const double gamma2 = 1. / (1 - vx * vx - vy * vy - vz * vz);
  const double p = eos_p4(E, e, nb, nq, ns);
  Q[0 * N + i] = tau * (e + p * (vx * vx + vy * vy + vz * vz)) * gamma2;
  Q[1 * N + i] = tau * (e + p) * vx * gamma2;
  Q[2 * N + i] = tau * (e + p) * vy * gamma2;
  Q[3 * N + i] = tau * (e + p) * vz * gamma2;
  Q[4 * N + i] = tau * nb * sqrt(gamma2);
  Q[5 * N + i] = tau * nq * sqrt(gamma2);
  Q[6 * N + i] = tau * ns * sqrt(gamma2);
}

/* A fresh Fluid's cells (Cell::Cell, src/cll.cpp:33-52) */
static void fresh_cells(const or_grid *g, or_state *s) {
  const long N = (long)g->nx * g->ny * g->nz;
  memset(s->Q, 0, sizeof(double) * 7 * N);
  memset(s->Qh, 0, sizeof(double) * 7 * N);
  memset(s->Qprev, 0, sizeof(double) * 7 * N);
  memset(s->pi, 0, sizeof(double) * 10 * N);
  memset(s->piH, 0, sizeof(double) * 10 * N);
  memset(s->Pi, 0, sizeof(double) * N);
  memset(s->PiH, 0, sizeof(double) * N);
  memset(s->m, 0, sizeof(double) * 3 * N);
  for (long i = 0; i < N; i++) s->vcc[i] = 1.;
}

static void set_all_m(or_state *s, long N, long i, double v) {
  s->m[i] = s->m[N + i] = s->m[2 * N + i] = v;
}

/* The collision-energy dependent longitudinal parameters that both readers
 * recompute per event at 27 GeV from the event's participant count
 * (src/icGlissando.cpp:188-195, src/icTrento.cpp:242-253) */
static void rhic27_update(or_ic_setup *u, int npart) {
  if (u->sNN == 27) {
    const double cent = (double)npart / (2. * 197.);
    u->eta0 = 0.888 - 0.213 * cent;
    u->sigEta = 1.088 - 0.213 * cent;
    u->neta0 = 1.332 - 0.319 * cent;
    u->nsigma = 0.788 - 0.213 * cent;
  }
}

/* per eta cell: evaluated with the C library in both arms */
static double f_eta(const or_ic_setup *u, double eta) {
  double fEta = 0.;
  if (fabs(eta) < u->eta0)
    fEta = 1.0;
  else if (fabs(eta) < u->ybeam)
    fEta = exp(-0.5 * pow((fabs(eta) - u->eta0) / u->sigEta, 2));
  return fEta;
}

/* setNormalization and setBaryonNorm iterated to |change| <= 1e-4, as both
 * constructors do (src/icGlissando.cpp:164-181, src/icTrento.cpp:185-202);
 * sdiv: the extra division of rho by dx dy of IcGlissando */
static void normalise(const or_grid *g, const or_ic_setup *u, double tau0, const double *rho,
                      const double *nrho, int nevents, int npart, int sdiv, int baryon, int cr,
                      double *sNorm, double *nNorm) {
  const double dx = gdx(g), dy = gdy(g), dz = gdz(g);
  double old;
  *sNorm = 1.0;
  do {
    old = *sNorm;
    double total_energy = 0.0;
    for (int ix = 0; ix < g->nx; ix++)
      for (int iy = 0; iy < g->ny; iy++)
        for (int iz = 0; iz < g->nz; iz++) {
          const long i = ix + (long)g->nx * (iy + (long)g->ny * iz);
          const double sv = sdiv ? *sNorm * rho[i] / nevents / dx / dy : *sNorm * rho[i] / nevents;
          const double e = or_s95p_e(sv, cr);
          const double eta = g->zmin + iz * dz;
          const double coshEta = cosh(eta);
          total_energy += tau0 * e * dx * dy * dz * coshEta;
        }
    *sNorm = pow(npart * 0.5 * u->sNN / total_energy, 0.75) * old;
  } while (fabs(*sNorm - old) > 0.0001);
  if (!baryon) return;
  *nNorm = 1.0;
  do {
    old = *nNorm;
    double Nb = 0.0;
    for (int ix = 0; ix < g->nx; ix++)
      for (int iy = 0; iy < g->ny; iy++)
        for (int iz = 0; iz < g->nz; iz++) {
          const long i = ix + (long)g->nx * (iy + (long)g->ny * iz);
          const double nb = *nNorm * nrho[i] / nevents / dx / dy / dz;
          Nb += nb * tau0 * dx * dy * dz;
        }
    *nNorm = npart / Nb * old;
  } while (fabs(*nNorm - old) > 0.0001);
}

/* the common setIC of IcGlissando and IcTrento (src/icGlissando.cpp:231-244,
 * src/icTrento.cpp:283-296): no saveQprev, so Qprev stays zero */
static void set_ic_common(const or_grid *g, const or_eos *E, const or_ic_setup *u, double tau0,
                          const double *rho, const double *nrho, int nevents, int sdiv,
                          double sNorm, double nNorm, int cr, or_state *s) {
  const long N = (long)g->nx * g->ny * g->nz;
  const double dx = gdx(g), dy = gdy(g), dz = gdz(g);
  for (int ix = 0; ix < g->nx; ix++)
    for (int iy = 0; iy < g->ny; iy++)
      for (int iz = 0; iz < g->nz; iz++) {
        const long i = ix + (long)g->nx * (iy + (long)g->ny * iz);
        const double sv = sdiv ? sNorm * rho[i] / nevents / dx / dy : sNorm * rho[i] / nevents;
        const double e = or_s95p_e(sv, cr);
        const double nb = u->sNN < 100 ? nNorm * nrho[i] / nevents / dx / dy / dz : 0.;
        const double x = g->xmin + ix * dx, eta = g->zmin + iz * dz;
        const double ueta = tanh(u->A * x) * sinh(u->ybeam - fabs(eta));
        const double u0 = sqrt(1.0 + ueta * ueta);
        set_prim_var(E, s->Q, N, i, tau0, e, nb, 0.4 * nb, 0., 0., 0., ueta / u0);
        if (e > 0.) set_all_m(s, N, i, 1.);
      }
}

int or_ic_glissando(const or_grid *g, const or_eos *E, const or_ic_setup *setup, double tau0,
                    const double *X, const double *Y, const int *C, const int *npart,
                    int nevents, int cr, or_state *s, double *norms) {
  const long N = (long)g->nx * g->ny * g->nz;
  const double dx = gdx(g), dy = gdy(g), dz = gdz(g);
  or_ic_setup u = *setup;
  const int ns = (int)(3.0 * u.Rg / dx);
  double *rho = calloc(N, sizeof(double)), *nrho = calloc(N, sizeof(double));
  if (!rho || !nrho) {
    free(rho);
    free(nrho);
    return -1;
  }
  fresh_cells(g, s);
  long base = 0, np_tot = 0;
  for (int ev = 0; ev < nevents; ev++) {
    rhic27_update(&u, npart[ev]);
    /* makeSmoothTable, src/icGlissando.cpp:187-228 */
    for (int ip = 0; ip < npart[ev]; ip++) {
      const double xp = X[base + ip], yp = Y[base + ip];
      const int cp = C[base + ip];
      const int ixc = (int)((xp - g->xmin) / dx);
      const int iyc = (int)((yp - g->ymin) / dy);
      const double norm_gauss = 2.0 * OR_C_PI * u.Rg * u.Rg;
      for (int ix = ixc - ns; ix < ixc + ns + 1; ix++)
        for (int iy = iyc - ns; iy < iyc + ns + 1; iy++)
          if (ix > 0 && ix < g->nx && iy > 0 && iy < g->ny) {
            const double xdiff = xp - (g->xmin + ix * dx);
            const double ydiff = yp - (g->ymin + iy * dy);
            double trSmear = 1.0 / norm_gauss *
                             xexp(-xdiff * xdiff / (2. * u.Rg * u.Rg) -
                                      ydiff * ydiff / (2. * u.Rg * u.Rg),
                                  cr);
            if (trSmear != trSmear || fabs(trSmear) > DBL_MAX) trSmear = 0.0;
            for (int iz = 0; iz < g->nz; iz++) {
              const long i = ix + (long)g->nx * (iy + (long)g->ny * iz);
              const double eta = g->zmin + iz * dz;
              double tilt = cp > 0 ? 0.5 * (u.etaM + eta) / u.etaM : 0.5 * (u.etaM - eta) / u.etaM;
              tilt = fmax(0.0, tilt);
              tilt = fmin(1.0, tilt);
              double bg = 0.;
              if (u.sNN < 100) {
                bg = cp > 0 ? exp(-pow(eta - u.neta0, 2) / (2. * u.nsigma * u.nsigma))
                            : exp(-pow(eta + u.neta0, 2) / (2. * u.nsigma * u.nsigma));
                bg /= u.nsigma * sqrt(2 * OR_C_PI);
              }
              const double fEta = f_eta(&u, eta);
              rho[i] += trSmear * fEta * tilt * ((1.0 - u.alphaMix) + abs(cp) * u.alphaMix);
              if (u.sNN < 100) nrho[i] += trSmear * ((1.0 - u.alphaMix) + abs(cp) * u.alphaMix) * bg;
            }
          }
    }
    base += npart[ev];
    np_tot += npart[ev];
  }
  double sNorm = 1., nNorm = 0.;
  normalise(g, &u, tau0, rho, nrho, nevents, (int)(np_tot / nevents), 1, u.sNN < 100, cr,
            &sNorm, &nNorm);
  set_ic_common(g, E, &u, tau0, rho, nrho, nevents, 1, sNorm, nNorm, cr, s);
  if (norms) {
    norms[0] = sNorm;
    norms[1] = nNorm;
  }
  free(rho);
  free(nrho);
  return 0;
}

/* IcTrento::interpolateGrid, src/icTrento.cpp:221-240: bilinear on the
 * event's n x n grid over [-xmaxG, xmaxG]^2, src[iy * n + ix] (file order) */
static double trento_interp(const double *src, int n, double xmaxG, double x, double y) {
  const double xminG = -xmaxG, yminG = -xmaxG, ymaxG = xmaxG;
  const double dxG = (xmaxG - xminG) / (n - 1);
  const double dyG = (ymaxG - yminG) / (n - 1);
  int ix = (int)((x - xminG) / dxG);
  int iy = (int)((y - yminG) / dyG);
  if (ix < 0) ix = 0;
  if (iy < 0) iy = 0;
  if (ix > n - 2) ix = n - 2;
  if (iy > n - 2) iy = n - 2;
  const double xm = x - xminG - ix * dxG;
  const double ym = y - yminG - iy * dyG;
  const double wx[2] = {1. - xm / dxG, xm / dxG};
  const double wy[2] = {1. - ym / dyG, ym / dyG};
  double r = 0.;
  for (int jx = 0; jx < 2; jx++)
    for (int jy = 0; jy < 2; jy++) r += wx[jx] * wy[jy] * src[(long)(iy + jy) * n + ix + jx];
  return fmax(r, 0.);
}

int or_ic_trento(const or_grid *g, const or_eos *E, const or_ic_setup *setup, double tau0,
                 const double *src, const int *ngrid, const double *gmax, const int *npart,
                 int nevents, int cr, or_state *s, double *norms) {
  const long N = (long)g->nx * g->ny * g->nz;
  const double dx = gdx(g), dy = gdy(g), dz = gdz(g);
  or_ic_setup u = *setup;
  double *rho = calloc(N, sizeof(double)), *nrho = calloc(N, sizeof(double));
  if (!rho || !nrho) {
    free(rho);
    free(nrho);
    return -1;
  }
  fresh_cells(g, s);
  long base = 0;
  for (int ev = 0; ev < nevents; ev++) {
    const int n = ngrid[ev];
    rhic27_update(&u, npart[ev]);
    /* makeSmoothTable, src/icTrento.cpp:242-275 */
    for (int ix = 0; ix < g->nx; ix++)
      for (int iy = 0; iy < g->ny; iy++)
        for (int iz = 0; iz < g->nz; iz++) {
          const long i = ix + (long)g->nx * (iy + (long)g->ny * iz);
          const double x = g->xmin + ix * dx, y = g->ymin + iy * dy, eta = g->zmin + iz * dz;
          if (u.sNN < 100) {
            double bg = eta > 0 ? exp(-pow(eta - u.neta0, 2) / (2. * u.nsigma * u.nsigma))
                                : exp(-pow(eta + u.neta0, 2) / (2. * u.nsigma * u.nsigma));
            bg /= u.nsigma * sqrt(2 * OR_C_PI);
            nrho[i] += trento_interp(src + base, n, gmax[ev], x, y) * bg;
          }
          rho[i] += trento_interp(src + base, n, gmax[ev], x, y) * f_eta(&u, eta);
        }
    base += (long)n * n;
  }
  double sNorm = 1., nNorm = 0.;
  if (u.sNN < 2760)
    normalise(g, &u, tau0, rho, nrho, nevents, npart[nevents - 1], 0, u.sNN < 100, cr, &sNorm,
              &nNorm);
  set_ic_common(g, E, &u, tau0, rho, nrho, nevents, 0, sNorm, nNorm, cr, s);
  if (norms) {
    norms[0] = sNorm;
    norms[1] = nNorm;
  }
  free(rho);
  free(nrho);
  return 0;
}

void or_ic_gubser(const or_grid *g, const or_eos *E, double tau, int cr, or_state *s) {
  const long N = (long)g->nx * g->ny * g->nz;
  const double dx = gdx(g), dy = gdy(g);
  fresh_cells(g, s);
  /* ICGubser::setIC, src/icGubser.cpp:17-60 (q = 1, t = 1) */
  for (int ix = 0; ix < g->nx; ix++)
    for (int iy = 0; iy < g->ny; iy++)
      for (int iz = 0; iz < g->nz; iz++) {
        const long i = ix + (long)g->nx * (iy + (long)g->ny * iz);
        const double x = g->xmin + ix * dx, y = g->ymin + iy * dy;
        const double _t = 1.0, q = 1.0;
        const double r = sqrt(x * x + y * y);
        const double _k = 2. * q * q * _t * r / (1. + q * q * _t * _t + q * q * r * r);
        double e = 4. * q * q /
                   (1. + 2. * q * q * (_t * _t + r * r) + xsq(q * q * (_t * _t - r * r), cr)) / _t;
        if (e < 0.) e = 0.;
        e = xpow(e, 4. / 3., cr);
        const double vx = x / (r + 1e-50) * _k, vy = y / (r + 1e-50) * _k;
        set_prim_var(E, s->Q, N, i, tau, e, 0., 0., 0., vx, vy, 0.);
        for (int k = 0; k < 7; k++) s->Qprev[k * N + i] = s->Q[k * N + i];
        if (e > 0.) set_all_m(s, N, i, 1.);
      }
}

void or_ic_table(const or_grid *g, const or_eos *E, double tau, int NX, int NY,
                 const double *xs, const double *ys, const double *val, double factor,
                 int glauber_var, int cr, or_state *s) {
  const long N = (long)g->nx * g->ny * g->nz;
  const double dx = gdx(g), dy = gdy(g), dz = gdz(g);
  fresh_cells(g, s);
  /* s95p::loadSongIC, src/s95p.cpp:43-66: val[ix * NY + iy] */
  double *t = malloc(sizeof(double) * (size_t)NX * NY);
  if (!t) return;
  for (long k = 0; k < (long)NX * NY; k++)
    t[k] = glauber_var == 1 ? or_s95p_e(factor * val[k], cr) : factor * val[k];
  const double xmin = xs[0], xmax = xs[NX - 1], ymin = ys[0], ymax = ys[NY - 1];
  /* IC::setIC, src/ic.cpp:18-55, with s95p::getSongEps, src/s95p.cpp:68-86 */
  for (int ix = 0; ix < g->nx; ix++)
    for (int iy = 0; iy < g->ny; iy++)
      for (int iz = 0; iz < g->nz; iz++) {
        const long i = ix + (long)g->nx * (iy + (long)g->ny * iz);
        const double x = g->xmin + ix * dx, y = g->ymin + iy * dy, eta = g->zmin + iz * dz;
        const double eta1 = fabs(eta) < 1.3 ? 0.0 : fabs(eta) - 1.3;
        const double etaFactor = exp(-eta1 * eta1 / 2.1 / 2.1) * (fabs(eta) < 5.3 ? 1.0 : 0.0);
        const double sdx = (xmax - xmin) / (NX - 1), sdy = (ymax - ymin) / (NY - 1);
        const int jx = (int)((x - xmin) / sdx), jy = (int)((y - ymin) / sdy);
        double eps = 0.0;
        if (!(jx < 0 || jx > NX - 2 || jy < 0 || jy > NY - 2)) {
          const double sx = x - xmin - jx * sdx, sy = y - ymin - jy * sdy;
          const double wx[2] = {(1. - sx / sdx), sx / sdx};
          const double wy[2] = {(1. - sy / sdy), sy / sdy};
          for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) eps += wx[a] * wy[b] * t[(long)(jx + a) * NY + jy + b];
        }
        double e = eps * etaFactor;
        if (e < 0.5) e = 0.0;
        set_prim_var(E, s->Q, N, i, tau, e, 0., 0., 0., 0., 0., 0.);
        for (int k = 0; k < 7; k++) s->Qprev[k * N + i] = s->Q[k * N + i];
        if (e > 0.) set_all_m(s, N, i, 1.);
      }
  free(t);
}

/* IcPartUrqmd (src/icPartUrqmd.cpp:17-253), icModel 3: each particle's
 * energy-momentum, baryon number and charge smeared over a 3D Gaussian
 * stencil normalised to its own sum (makeSmoothTable, :105-175), summed over
 * the events; then per cell transformPV of the averaged Q, a cut, setPrimVar
 * and setAllM (setIC, :202-227).  p[n][8] = tau, x, y, eta, mt, px, py, rap.
 * The per-particle cosh / sinh of (rap - eta + zdiff) and gamma_z use the C
 * library in both arms (the CUDA path's host side computes them). */
void or_ic_urqmd(const or_grid *g, const or_eos *E, double tau0, const double *p,
                 const int *id, const int *charge, const int *npart, int nevents, double Rgt,
                 double Rgz, int cr, or_state *s) {
  const long N = (long)g->nx * g->ny * g->nz;
  const double dx = gdx(g), dy = gdy(g), dz = gdz(g);
  const double Rgx = Rgt, Rgy = Rgt;
  const int nsx = (int)(6.0 * Rgx / dx), nsy = (int)(6.0 * Rgy / dy);
  const int nsz = (int)(1.5 * Rgz / dz);
  double *T = calloc(6 * (size_t)N, sizeof(double)); /* T00, T0x, T0y, T0z, QB, QE */
  if (!T) return;
  fresh_cells(g, s);
  long np = 0;
  for (int ev = 0; ev < nevents; ev++) np += npart[ev];
  for (long ip = 0; ip < np; ip++) {
    const double *q = p + 8 * ip;
    const double X = q[1], Y = q[2], Eta = q[3], Mt = q[4], Px = q[5], Py = q[6], Rap = q[7];
    const int ixc = (int)round((X - g->xmin) / dx);
    const int iyc = (int)round((Y - g->ymin) / dy);
    const int izc = (int)round((Eta - g->zmin) / dz);
    const double gammaz = cosh(Rap - Eta);
    double norm_gauss = 0.0;
    for (int pass = 0; pass < 2; pass++)
      for (int ix = ixc - nsx; ix < ixc + nsx + 1; ix++)
        for (int iy = iyc - nsy; iy < iyc + nsy + 1; iy++)
          for (int iz = izc - nsz; iz < izc + nsz + 1; iz++)
            if (ix > 0 && ix < g->nx && iy > 0 && iy < g->ny && iz > 0 && iz < g->nz) {
              const double xdiff = X - (g->xmin + ix * dx);
              const double ydiff = Y - (g->ymin + iy * dy);
              const double zdiff = Eta - (g->zmin + iz * dz);
              double a;
              if (fabs(Rgz) < 1e-5)
                a = -xdiff * xdiff / Rgx / Rgx - ydiff * ydiff / Rgy / Rgy;
              else
                a = -xdiff * xdiff / Rgx / Rgx - ydiff * ydiff / Rgy / Rgy -
                    zdiff * zdiff / Rgz / Rgz * gammaz * gammaz * tau0 * tau0;
              if (pass == 0) {
                norm_gauss += xexp(a, cr);
                continue;
              }
              double weight = 1.0 / norm_gauss * xexp(a, cr);
              if (weight != weight || fabs(weight) > DBL_MAX) weight = 0.0;
              const long i = ix + (long)g->nx * (iy + (long)g->ny * iz);
              T[0 * N + i] += weight * Mt * cosh(Rap - Eta + zdiff);
              T[1 * N + i] += weight * Px;
              T[2 * N + i] += weight * Py;
              T[3 * N + i] += weight * Mt * sinh(Rap - Eta + zdiff);
              if (id[ip] > 0 && id[ip] < 56) T[4 * N + i] += weight;
              if (id[ip] < 0 && id[ip] > -56) T[4 * N + i] -= weight;
              T[5 * N + i] += charge[ip] * weight;
            }
  }
  for (int ix = 0; ix < g->nx; ix++)
    for (int iy = 0; iy < g->ny; iy++)
      for (int iz = 0; iz < g->nz; iz++) {
        const long i = ix + (long)g->nx * (iy + (long)g->ny * iz);
        double Q[7], o[8];
        for (int k = 0; k < 6; k++) Q[k] = T[k * N + i] / nevents / dx / dy / dz / tau0;
        Q[6] = 0.0;
        or_transform_pv(E, Q, 1, o);
        double e = o[0], nb = o[2], nq = o[3], ns = o[4], vx = o[5], vy = o[6], vz = o[7];
        const double x = g->xmin + ix * dx, y = g->ymin + iy * dy, eta = g->zmin + iz * dz;
        if (e < 1e-7 || fabs(x) > 10. || fabs(y) > 10. || fabs(eta) > 5.) {
          e = nb = nq = 0.0;
          vx = vy = vz = 0.0;
        }
        set_prim_var(E, s->Q, N, i, tau0, e, nb, nq, ns, vx, vy, vz);
        if (e > 0.) set_all_m(s, N, i, 1.);
      }
  free(T);
}
