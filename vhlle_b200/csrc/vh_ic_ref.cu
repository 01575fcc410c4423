// vh_ic_ref.cu -- the reference's initial-state modules on the device:
// IcGlissando (vh_init_glissando), IcTrento (vh_init_trento), ICGubser
// (vh_init_gubser) and IC over the s95p table (vh_init_table), the modules
// the driver picks by icModel 5, 7, 4 and 2 (src/main.cpp:324-366).
//
// What costs on the host is per cell or per source: a GLISSANDO event's
// few hundred sources each smeared over ~170 transverse cells times every
// eta cell, a TRENTO grid interpolated at every cell per event, and the
// s95p entropy-to-energy inversion (a Newton iteration of five powers per
// step) of every cell once per normalisation pass and once more at the end.
// Those run here:
//
//   k_gliss_rho   one thread per transverse cell and 8 eta cells: the
//                 sources in file order (staged through shared memory),
//                 each within its +-ns stencil adding the reference's
//                 trSmear fEta tilt w (and the baryon term) in the order
//                 the host loop adds them, so every cell's sum is the
//                 reference's bit for bit
//   k_trento_rho  the same thread shape over the events' grids
//   k_ic_terms    a normalisation pass's per-cell terms (s95p_e and the
//                 cell's energy, or its baryon number), written in the
//                 reference's loop order (ix, iy, iz)
//   k_seq_sum     their sum in that order, one thread adding tiles that
//                 the block's other warps stage in shared memory: the same
//                 rounded sum as the host loop
//   k_ic_set      e = s95p_e(..), nb, setPrimVar, setAllM for every cell
//   k_ic_gubser, k_table_prep, k_ic_table   the other two modules
//
// The normalisation's update sNorm = (npart sNN / 2 / E)^(3/4) sNorm_old and
// its stopping test run on the host between passes (one 8-byte copy each),
// with the C library's pow as the reference.  Per-axis factors (the
// rapidity profiles of each event, cosh(eta), the shear-flow velocity
// tanh(A x) sinh(ybeam - |eta|)) are nz or nx*nz values computed on the
// host with the C library.  exp and pow on the device are the correctly
// rounded crm::exp_cr / crm::pow_cr; the reference's C library misrounds
// pow by one ulp in about one call in a thousand, so single cells can
// differ from the reference in the last bits.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/vhlle_b200.h"
#include "vh_crmath.cuh"
#include "vh_ctx.cuh"
#include "vh_physics.cuh"

namespace vh {
namespace icr {

constexpr double kCPi = 3.14159265358979312;  // C_PI, src/inc.h:18
constexpr int kTpb = 128;
constexpr int kKz = 8;             // eta cells per thread in the source sums
constexpr int kS95pMaxIt = 200;    // the reference iterates without a bound
constexpr int kNormMaxIt = 10000;  // likewise its normalisation loops

// x^y and e^x kept out of line: s95p_s holds up to six powers and two
// exponentials, each ~800 FP64 operations inlined, and the Newton loop
// around it would otherwise be tens of KB of straight-line code per kernel
__device__ __noinline__ double pw(double x, double y) { return crm::pow_cr(x, y); }
__device__ __noinline__ double ex(double x) { return crm::exp_cr(x); }

// s95p::s95p_s, src/s95p.cpp:14-32 (the s95p-PCE fit of s(e))
__device__ double s95p_s(double e) {
  double val;
  if (e < 0.1270769021427449)
    val = 12.2304 * pw(e, 1.16849);
  else if (e < 0.4467079524674040)
    val = 11.9279 * pw(e, 1.15635);
  else if (e < 1.9402832534193788)
    val = 0.0580578 + 11.833 * pw(e, 1.16187);
  else if (e < 3.7292474570977285)
    val = 18.202 * e - 62.021814 - 4.85479 * ex(-2.72407e-11 * pw(e, 4.54886)) +
          65.1272 * pw(e, -0.128012) * ex(-0.00369624 * pw(e, 1.18735)) -
          4.75253 * pw(e, -1.18423);
  else
    val = 18.202 * e - 63.0218 - 4.85479 * ex(-2.72407e-11 * pw(e, 4.54886)) +
          65.1272 * pw(e, -0.128012) * ex(-0.00369624 * pw(e, 1.18735));
  return pw(val, 3. / 4.);
}

// s95p::s95p_e, src/s95p.cpp:34-41; *bad gets bit 1 if kS95pMaxIt steps
// did not converge (the reference would not return)
__device__ double s95p_e(double s, unsigned* bad) {
  double e = pw(s, 4. / 3.) / 18.2, e0;
  int it = 0;
  do {
    e0 = e;
    e = e0 - (s95p_s(e0) - s) / (6.608681233 * pw(e0, -0.25));
    if (++it > kS95pMaxIt) {
      atomicOr(bad, 1u);
      break;
    }
  } while (fabs(e - e0) > 1e-10);
  return e;
}

// Cell::setPrimVar, src/cll.cpp:222-241 (EoS::p at (e, nb); the kinds whose
// p also depends on nq are evaluated at nq = 0 here, which only matters with
// a non-zero velocity)
__device__ void set_prim(const EosDev& E, double tau, double e, double nb, double nq, double ns,
                         double vx, double vy, double vz, double q[7]) {
  const double gamma2 = 1. / (1 - vx * vx - vy * vy - vz * vz);
  const double p = eos_p<EK_ANY>(E, e, nb);
  q[0] = tau * (e + p * (vx * vx + vy * vy + vz * vz)) * gamma2;
  q[1] = tau * (e + p) * vx * gamma2;
  q[2] = tau * (e + p) * vy * gamma2;
  q[3] = tau * (e + p) * vz * gamma2;
  q[4] = tau * nb * sqrt(gamma2);
  q[5] = tau * nq * sqrt(gamma2);
  q[6] = tau * ns * sqrt(gamma2);
}

// a fresh Fluid's cell (src/cll.cpp:33-52) after setPrimVar, saveQprev when
// qprev, and setAllM(m)
__device__ void put_cell(const Fields& f, long long N, long long i, const double q[7], bool qprev,
                         double m) {
#pragma unroll
  for (int k = 0; k < 7; k++) {
    f.Q[k * N + i] = q[k];
    f.Qprev[k * N + i] = qprev ? q[k] : 0.;
    f.Qh[k * N + i] = 0.;
  }
#pragma unroll
  for (int k = 0; k < 10; k++) {
    f.pi[k * N + i] = 0.;
    f.piH[k * N + i] = 0.;
  }
  f.Pi[i] = 0.;
  f.PiH[i] = 0.;
  f.vcc[i] = 1.;
#pragma unroll
  for (int k = 0; k < 3; k++) f.m[k * N + i] = m;
}

struct ColGeo {
  int nx, ny, nz;
  double xmin, ymin, dx, dy;
};

struct GlissArgs {
  ColGeo g;
  int ns;          // (int)(3 Rg / dx), src/icGlissando.cpp:125
  double Rg, alphaMix;
  int baryon;      // sNN < 100
  const double *sx, *sy;
  const int *sc, *sev;  // code and event of each source
  int nsrc;
  const double* fEta;   // [nev][nz]
  const double* tilt;   // [2][nz] (code > 0, else)
  const double* bg;     // [nev][2][nz] baryon Gaussian / (nsigma sqrt(2 pi))
  double *rho, *nrho;   // [N] grid order
};

// IcGlissando::makeSmoothTable over every event, src/icGlissando.cpp:187-228
__global__ void __launch_bounds__(kTpb) k_gliss_rho(GlissArgs a) {
  __shared__ double shx[kTpb], shy[kTpb];
  __shared__ int shc[kTpb], she[kTpb];
  const ColGeo& g = a.g;
  const int ncol = g.nx * g.ny;
  const int nch = (g.nz + kKz - 1) / kKz;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = t < (long long)ncol * nch;
  const int col = in ? (int)(t % ncol) : 0, ch = in ? (int)(t / ncol) : 0;
  const int ix = col % g.nx, iy = col / g.nx;
  const bool open = in && ix > 0 && iy > 0;  // the loop's ix > 0 && iy > 0
  double r[kKz], nr[kKz];
#pragma unroll
  for (int k = 0; k < kKz; k++) r[k] = nr[k] = 0.0;
  const double norm_gauss = 2.0 * kCPi * a.Rg * a.Rg;
  const double inv_norm = 1.0 / norm_gauss;
  const double two_rg2 = 2. * a.Rg * a.Rg;
  const double xc = g.xmin + ix * g.dx, yc = g.ymin + iy * g.dy;
  for (int base = 0; base < a.nsrc; base += kTpb) {
    __syncthreads();
    const int k = base + threadIdx.x;
    if (k < a.nsrc) {
      shx[threadIdx.x] = a.sx[k];
      shy[threadIdx.x] = a.sy[k];
      shc[threadIdx.x] = a.sc[k];
      she[threadIdx.x] = a.sev[k];
    }
    __syncthreads();
    if (!open) continue;
    const int n = min(kTpb, a.nsrc - base);
    for (int j = 0; j < n; j++) {
      const double xs = shx[j], ys = shy[j];
      const int ixc = (int)((xs - g.xmin) / g.dx);
      const int iyc = (int)((ys - g.ymin) / g.dy);
      if (ix < ixc - a.ns || ix > ixc + a.ns || iy < iyc - a.ns || iy > iyc + a.ns) continue;
      const double xdiff = xs - xc, ydiff = ys - yc;
      double tr = inv_norm * crm::exp_cr(-xdiff * xdiff / two_rg2 - ydiff * ydiff / two_rg2);
      if (tr != tr || fabs(tr) > DBL_MAX) tr = 0.0;
      const int c = shc[j], ev = she[j];
      const double w = (1.0 - a.alphaMix) + abs(c) * a.alphaMix;
      const int sg = c > 0 ? 0 : 1;
      const double* fe = a.fEta + (long long)ev * g.nz;
      const double* tl = a.tilt + sg * g.nz;
      const double* bgp = a.bg + ((long long)ev * 2 + sg) * g.nz;
#pragma unroll
      for (int kz = 0; kz < kKz; kz++) {
        const int iz = ch * kKz + kz;
        if (iz < g.nz) {
          r[kz] += tr * fe[iz] * tl[iz] * w;
          if (a.baryon) nr[kz] += tr * w * bgp[iz];
        }
      }
    }
  }
  if (!in) return;
#pragma unroll
  for (int kz = 0; kz < kKz; kz++) {
    const int iz = ch * kKz + kz;
    if (iz < g.nz) {
      const long long i = col + (long long)ncol * iz;
      a.rho[i] = r[kz];
      a.nrho[i] = nr[kz];
    }
  }
}

// IcTrento::interpolateGrid, src/icTrento.cpp:221-240 (src[iy * n + ix])
__device__ double trento_interp(const double* __restrict__ src, int n, double xmaxG, double x,
                                double y) {
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
#pragma unroll
  for (int jx = 0; jx < 2; jx++)
#pragma unroll
    for (int jy = 0; jy < 2; jy++) r += wx[jx] * wy[jy] * src[(long long)(iy + jy) * n + ix + jx];
  return fmax(r, 0.);
}

struct TrentoArgs {
  ColGeo g;
  int baryon;
  const double* grid;
  const long long* goff;  // [nev] offset of each event's grid
  const int* gn;
  const double* gmax;
  int nev;
  const double* fEta;  // [nev][nz]
  const double* bgz;   // [nev][nz]
  double *rho, *nrho;
};

// IcTrento::makeSmoothTable over every event, src/icTrento.cpp:242-275
__global__ void __launch_bounds__(kTpb) k_trento_rho(TrentoArgs a) {
  const ColGeo& g = a.g;
  const int ncol = g.nx * g.ny;
  const int nch = (g.nz + kKz - 1) / kKz;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ncol * nch) return;
  const int col = (int)(t % ncol), ch = (int)(t / ncol);
  const int ix = col % g.nx, iy = col / g.nx;
  const double x = g.xmin + ix * g.dx, y = g.ymin + iy * g.dy;
  double r[kKz], nr[kKz];
#pragma unroll
  for (int k = 0; k < kKz; k++) r[k] = nr[k] = 0.0;
  for (int ev = 0; ev < a.nev; ev++) {
    const double v = trento_interp(a.grid + a.goff[ev], a.gn[ev], a.gmax[ev], x, y);
    const double* fe = a.fEta + (long long)ev * g.nz;
    const double* bg = a.bgz + (long long)ev * g.nz;
#pragma unroll
    for (int kz = 0; kz < kKz; kz++) {
      const int iz = ch * kKz + kz;
      if (iz < g.nz) {
        if (a.baryon) nr[kz] += v * bg[iz];
        r[kz] += v * fe[iz];
      }
    }
  }
#pragma unroll
  for (int kz = 0; kz < kKz; kz++) {
    const int iz = ch * kKz + kz;
    if (iz < g.nz) {
      const long long i = col + (long long)ncol * iz;
      a.rho[i] = r[kz];
      a.nrho[i] = nr[kz];
    }
  }
}

enum { TERM_E = 0, TERM_E_DXDY = 1, TERM_NB = 2 };

struct TermArgs {
  int nx, ny, nz;
  long long N;
  double dx, dy, dz, tau0;
  int mode;
  double norm, nev;
  const double* rho;
  const double* coshEta;  // [nz]
  double* terms;          // [N] in the order (ix, iy, iz), iz fastest
  unsigned* bad;
};

// One pass of setNormalization (src/icGlissando.cpp:317-331,
// src/icTrento.cpp:349-362) or setBaryonNorm (:333-346, :364-375): the
// cell's term of the sum
__global__ void __launch_bounds__(kTpb) k_ic_terms(TermArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const int nxy = a.nx * a.ny;
  const int iz = (int)(i / nxy), it = (int)(i % nxy);
  const int ix = it % a.nx, iy = it / a.nx;
  double term;
  if (a.mode == TERM_NB) {
    const double nb = a.norm * a.rho[i] / a.nev / a.dx / a.dy / a.dz;
    term = nb * a.tau0 * a.dx * a.dy * a.dz;
  } else {
    const double sv = a.mode == TERM_E_DXDY ? a.norm * a.rho[i] / a.nev / a.dx / a.dy
                                            : a.norm * a.rho[i] / a.nev;
    const double e = s95p_e(sv, a.bad);
    term = a.tau0 * e * a.dx * a.dy * a.dz * a.coshEta[iz];
  }
  a.terms[((long long)ix * a.ny + iy) * a.nz + iz] = term;
}

// sum of t[0..n) from 0.0 in index order, rounded after every addition as
// the host loop: thread 0 adds a tile of terms from shared memory while the
// block's loader warps stage the next tile, so the running sum waits only on
// its own additions.  Each loader warp keeps its 256 terms of the tile with
// the zeros squeezed out, in order (ballot and prefix count), and thread 0
// adds the warps' runs in warp order: the same sequence of non-zero
// additions as the host loop, whose zero terms change nothing (the running
// sum starts at +0 and is never -0, and s + (+-0) = s for every other s; the
// vacuum cells' terms are exactly zero).
constexpr int kSumLoaders = 8;                     // loader warps
constexpr int kSumThreads = 32 * (1 + kSumLoaders);
constexpr int kSumRun = 256;                       // terms per loader warp and tile
constexpr int kSumTile = kSumLoaders * kSumRun;    // 2 x 16 KB of shared memory

__global__ void __launch_bounds__(kSumThreads) k_seq_sum(const double* __restrict__ t, long long n,
                                                         double* __restrict__ out) {
  __shared__ double buf[2][kSumTile];
  __shared__ int cnt[2][kSumLoaders];
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const long long ntile = (n + kSumTile - 1) / kSumTile;
  // loader warp w stages terms [w * kSumRun, (w + 1) * kSumRun) of a tile
  auto stage = [&](long long tile, int b) {
    const int w = warp - 1;
    const long long base = tile * kSumTile + (long long)w * kSumRun;
    double* dst = buf[b] + w * kSumRun;
    int c = 0;
    for (int r = 0; r < kSumRun; r += 32) {
      const long long k = base + r + lane;
      const double v = k < n ? t[k] : 0.0;
      const unsigned live = __ballot_sync(0xffffffffu, v != 0.0);  // NaN counts
      if (v != 0.0) dst[c + __popc(live & ((1u << lane) - 1u))] = v;
      c += __popc(live);
    }
    if (lane == 0) cnt[b][w] = c;
  };
  if (warp > 0 && ntile > 0) stage(0, 0);
  __syncthreads();
  double s = 0.0;
  for (long long tile = 0; tile < ntile; tile++) {
    const int b = (int)(tile & 1);
    if (warp > 0 && tile + 1 < ntile) stage(tile + 1, b ^ 1);
    if (tid == 0)
      for (int w = 0; w < kSumLoaders; w++) {
        const double* p = buf[b] + w * kSumRun;
        const int m = cnt[b][w];
#pragma unroll 4
        for (int j = 0; j < m; j++) s += p[j];
      }
    __syncthreads();
  }
  if (tid == 0) out[0] = s;
}

struct SetArgs {
  int nx, ny, nz;
  long long N;
  double dx, dy, dz, tau0;
  int sdiv, baryon;
  double sNorm, nNorm, nev;
  const double *rho, *nrho;
  const double* vz;  // [nz][nx] u^eta / u^tau of the shear flow
  EosDev E;
  Fields f;
  unsigned* bad;
};

// the common setIC of IcGlissando and IcTrento (src/icGlissando.cpp:231-244,
// src/icTrento.cpp:283-296): no saveQprev
__global__ void __launch_bounds__(kTpb) k_ic_set(SetArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const int nxy = a.nx * a.ny;
  const int iz = (int)(i / nxy), ix = (int)(i % nxy) % a.nx;
  const double sv = a.sdiv ? a.sNorm * a.rho[i] / a.nev / a.dx / a.dy : a.sNorm * a.rho[i] / a.nev;
  const double e = s95p_e(sv, a.bad);
  const double nb = a.baryon ? a.nNorm * a.nrho[i] / a.nev / a.dx / a.dy / a.dz : 0.;
  double q[7];
  set_prim(a.E, a.tau0, e, nb, 0.4 * nb, 0., 0., 0., a.vz[(long long)iz * a.nx + ix], q);
  put_cell(a.f, a.N, i, q, false, e > 0. ? 1. : 0.);
}

// ICGubser::setIC, src/icGubser.cpp:17-60 (q = 1, t = 1)
__global__ void __launch_bounds__(kTpb) k_ic_gubser(Geo g, double xmin, double ymin, double tau,
                                                     EosDev E, Fields f) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const int nxy = g.nx * g.ny;
  const int it = (int)(i % nxy);
  const int ix = it % g.nx, iy = it / g.nx;
  const double x = xmin + ix * g.dx, y = ymin + iy * g.dy;
  const double _t = 1.0, q = 1.0;
  const double r = sqrt(x * x + y * y);
  const double _k = 2. * q * q * _t * r / (1. + q * q * _t * _t + q * q * r * r);
  const double d = q * q * (_t * _t - r * r);
  double e = 4. * q * q / (1. + 2. * q * q * (_t * _t + r * r) + d * d) / _t;  // pow(d, 2)
  if (e < 0.) e = 0.;
  e = crm::pow_cr(e, 4. / 3.);
  const double vx = x / (r + 1e-50) * _k, vy = y / (r + 1e-50) * _k;
  double qv[7];
  set_prim(E, tau, e, 0., 0., 0., vx, vy, 0., qv);
  put_cell(f, g.N, i, qv, true, e > 0. ? 1. : 0.);
}

// s95p::loadSongIC's conversion of the table, src/s95p.cpp:55-59
__global__ void __launch_bounds__(kTpb) k_table_prep(const double* __restrict__ val, long long n,
                                                      double factor, int glauber_var,
                                                      double* __restrict__ out, unsigned* bad) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  out[k] = glauber_var == 1 ? s95p_e(factor * val[k], bad) : factor * val[k];
}

struct TableArgs {
  Geo g;
  double xmin, ymin, tau;
  int NX, NY;
  double txmin, txmax, tymin, tymax;
  const double* t;     // [NX][NY] converted table
  const double* etaF;  // [nz] the rapidity factor
  EosDev E;
  Fields f;
};

// IC::setIC, src/ic.cpp:18-55, with s95p::getSongEps, src/s95p.cpp:68-86
__global__ void __launch_bounds__(kTpb) k_ic_table(TableArgs a) {
  const Geo& g = a.g;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const int nxy = g.nx * g.ny;
  const int iz = (int)(i / nxy), it = (int)(i % nxy);
  const int ix = it % g.nx, iy = it / g.nx;
  const double x = a.xmin + ix * g.dx, y = a.ymin + iy * g.dy;
  const double sdx = (a.txmax - a.txmin) / (a.NX - 1), sdy = (a.tymax - a.tymin) / (a.NY - 1);
  const int jx = (int)((x - a.txmin) / sdx), jy = (int)((y - a.tymin) / sdy);
  double eps = 0.0;
  if (!(jx < 0 || jx > a.NX - 2 || jy < 0 || jy > a.NY - 2)) {
    const double sx = x - a.txmin - jx * sdx, sy = y - a.tymin - jy * sdy;
    const double wx[2] = {(1. - sx / sdx), sx / sdx};
    const double wy[2] = {(1. - sy / sdy), sy / sdy};
#pragma unroll
    for (int p = 0; p < 2; p++)
#pragma unroll
      for (int q = 0; q < 2; q++) eps += wx[p] * wy[q] * a.t[(long long)(jx + p) * a.NY + jy + q];
  }
  double e = eps * a.etaF[iz];
  if (e < 0.5) e = 0.0;
  double qv[7];
  set_prim(a.E, a.tau, e, 0., 0., 0., 0., 0., 0., qv);
  put_cell(a.f, g.N, i, qv, true, e > 0. ? 1. : 0.);
}

// ---- IcPartUrqmd (src/icPartUrqmd.cpp:105-175, 202-227)
constexpr int kUqTx = 32, kUqTy = 4;  // transverse tile of one block (one eta cell)

struct UrqmdArgs {
  Geo g;
  double xmin, ymin, zmin, tau0, Rgx, Rgy, Rgz, nev;
  int nsx, nsy, nsz;
  const double* p;    // [n][8] tau, x, y, eta, mt, px, py, rap
  const int* id;
  const int* charge;
  const int* c3;      // [n][3] ixc, iyc, izc
  const double* gz;   // [n] gamma_z = cosh(rap - eta)
  const double* csh;  // [n][2 nsz + 1][2] cosh, sinh of (rap - eta + zdiff) per stencil plane
  double* norm;       // [n]
  int n;
  const int* toff;    // [ntiles + 1] CSR of the particles whose stencil meets a tile
  const int* tlist;
  int ntx;
  double* T;          // [6][N] T00, T0x, T0y, T0z, QB, QE
};

// the Gaussian's exponent, as both of the module's stencil loops write it
__device__ __forceinline__ double uq_arg(const UrqmdArgs& a, double xdiff, double ydiff,
                                         double zdiff, double gammaz) {
  if (fabs(a.Rgz) < 1e-5) return -xdiff * xdiff / a.Rgx / a.Rgx - ydiff * ydiff / a.Rgy / a.Rgy;
  return -xdiff * xdiff / a.Rgx / a.Rgx - ydiff * ydiff / a.Rgy / a.Rgy -
         zdiff * zdiff / a.Rgz / a.Rgz * gammaz * gammaz * a.tau0 * a.tau0;
}

// norm_gauss of every particle: its stencil in the module's loop order
__global__ void __launch_bounds__(kTpb) k_urqmd_norm(UrqmdArgs a) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= a.n) return;
  const Geo& g = a.g;
  const double X = a.p[8 * ip + 1], Y = a.p[8 * ip + 2], Eta = a.p[8 * ip + 3];
  const int ixc = a.c3[3 * ip], iyc = a.c3[3 * ip + 1], izc = a.c3[3 * ip + 2];
  const double gammaz = a.gz[ip];
  double s = 0.0;
  for (int ix = ixc - a.nsx; ix < ixc + a.nsx + 1; ix++)
    for (int iy = iyc - a.nsy; iy < iyc + a.nsy + 1; iy++)
      for (int iz = izc - a.nsz; iz < izc + a.nsz + 1; iz++)
        if (ix > 0 && ix < g.nx && iy > 0 && iy < g.ny && iz > 0 && iz < g.nz) {
          const double xdiff = X - (a.xmin + ix * g.dx);
          const double ydiff = Y - (a.ymin + iy * g.dy);
          const double zdiff = Eta - (a.zmin + iz * g.dz);
          s += ex(uq_arg(a, xdiff, ydiff, zdiff, gammaz));
        }
  a.norm[ip] = s;
}

// every cell's sums over the particles whose stencil covers it, in file
// order (the tile's list is in that order)
__global__ void __launch_bounds__(kUqTx * kUqTy) k_urqmd_T(UrqmdArgs a) {
  const Geo& g = a.g;
  const int tile = blockIdx.x, iz = blockIdx.y;
  const int ix = (tile % a.ntx) * kUqTx + threadIdx.x % kUqTx;
  const int iy = (tile / a.ntx) * kUqTy + threadIdx.x / kUqTx;
  const bool in = ix < g.nx && iy < g.ny;
  const bool open = in && ix > 0 && iy > 0 && iz > 0;  // the loops' ix, iy, iz > 0
  double t00 = 0., t0x = 0., t0y = 0., t0z = 0., qb = 0., qe = 0.;
  if (open) {
    const double xc = a.xmin + ix * g.dx, yc = a.ymin + iy * g.dy, zc = a.zmin + iz * g.dz;
    for (int k = a.toff[tile]; k < a.toff[tile + 1]; k++) {
      const int ip = a.tlist[k];
      const int ixc = a.c3[3 * ip], iyc = a.c3[3 * ip + 1], izc = a.c3[3 * ip + 2];
      if (ix < ixc - a.nsx || ix > ixc + a.nsx || iy < iyc - a.nsy || iy > iyc + a.nsy ||
          iz < izc - a.nsz || iz > izc + a.nsz)
        continue;
      const double* q = a.p + 8 * ip;
      const double xdiff = q[1] - xc, ydiff = q[2] - yc, zdiff = q[3] - zc;
      double w = 1.0 / a.norm[ip] * ex(uq_arg(a, xdiff, ydiff, zdiff, a.gz[ip]));
      if (w != w || fabs(w) > DBL_MAX) w = 0.0;
      const double* cs = a.csh + ((long long)ip * (2 * a.nsz + 1) + (iz - (izc - a.nsz))) * 2;
      t00 += w * q[4] * cs[0];
      t0x += w * q[5];
      t0y += w * q[6];
      t0z += w * q[4] * cs[1];
      const int id = a.id[ip];
      if (id > 0 && id < 56) qb += w;
      if (id < 0 && id > -56) qb -= w;
      qe += a.charge[ip] * w;
    }
  }
  if (!in) return;
  const long long N = g.N, i = ix + (long long)g.nx * (iy + (long long)g.ny * iz);
  a.T[0 * N + i] = t00;
  a.T[1 * N + i] = t0x;
  a.T[2 * N + i] = t0y;
  a.T[3 * N + i] = t0z;
  a.T[4 * N + i] = qb;
  a.T[5 * N + i] = qe;
}

// IcPartUrqmd::setIC: transformPV of the averaged Q, the module's cut,
// setPrimVar, setAllM; no saveQprev
__global__ void __launch_bounds__(kTpb) k_urqmd_set(UrqmdArgs a, EosDev E, Fields f) {
  const Geo& g = a.g;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const long long N = g.N;
  const int nxy = g.nx * g.ny;
  const int iz = (int)(i / nxy), it = (int)(i % nxy);
  const int ix = it % g.nx, iy = it / g.nx;
  double Q[7];
#pragma unroll
  for (int k = 0; k < 6; k++) Q[k] = a.T[k * N + i] / a.nev / g.dx / g.dy / g.dz / a.tau0;
  Q[6] = 0.0;
  Prim o;
  transform_pv<EK_ANY>(E, Q, o);
  double e = o.e, nb = o.nb, nq = o.nq, vx = o.vx, vy = o.vy, vz = o.vz;
  const double x = a.xmin + ix * g.dx, y = a.ymin + iy * g.dy, eta = a.zmin + iz * g.dz;
  if (e < 1e-7 || fabs(x) > 10. || fabs(y) > 10. || fabs(eta) > 5.) {
    e = nb = nq = 0.0;
    vx = vy = vz = 0.0;
  }
  double q[7];
  set_prim(E, a.tau0, e, nb, nq, o.ns, vx, vy, vz, q);
  put_cell(f, N, i, q, false, e > 0. ? 1. : 0.);
}

}  // namespace icr
}  // namespace vh

// ---------------------------------------------------------------- host side
namespace {

using vh::icr::kTpb;

struct SetupEntry {
  int model;
  const char* name;
  vh_ic_setup s;  // sNN, eta0, sigEta, etaM, ybeam, alphaMix, Rg, A, nsigma, neta0
};

// The setups' constants as the two constructors set them
// (src/icGlissando.cpp:33-123, src/icTrento.cpp:33-88); what a setup leaves
// unset is 0 here and unused by the reference (the baryon Gaussian's below
// 100 GeV only; RHIC27's rapidity constants come from each event's npart).
const SetupEntry kSetups[] = {
    {5, "LHC276", {2760, 2.3, 1.4, 4, 7.98, 0.15, 0.4, 0.0, 0, 0}},
    {5, "RHIC200", {200, 1.5, 1.4, 3.36, 5.36, 0.145, 0.4, 0.0, 0.6, 1.4}},
    {5, "LHC5020", {5020, 3.7, 1.4, 4.5, 8.585, 0.15, 0.4, 0.0, 0, 0}},
    {5, "RHIC62", {62.4, 1.8, 0.7, 1.8, 4.2, 0.132, 0.4, 0.0, 1.0, 2.2}},
    {5, "AFTER72", {72, 1.8, 0.7, 1.8, 4.2, 0.132, 0.4, 0.0, 1.0, 2.2}},
    {5, "RHIC27", {27, 0, 0, 1.0, 3.36, 0.123, 0.4, 0.0, 0, 0}},
    {7, "LHC276", {2760, 2.3, 1.4, 4, 7.98, 0.15, 0.4, 0.0, 0, 0}},
    {7, "RHIC200", {200, 1.5, 1.4, 3.36, 5.36, 0.145, 0.4, 0.0, 0.6, 1.4}},
    {7, "LHC5020", {5020, 2.5, 1.4, 4, 7.98, 0.15, 0.4, 0.0, 0, 0}},
    {7, "RHIC62", {62.4, 1.8, 0.7, 1.8, 4.2, 0.132, 0.4, 0.0, 1.0, 2.2}},
    {7, "RHIC27", {27, 0, 0, 1.0, 3.36, 0.123, 0.4, 0.0, 0, 0}},
};

// device buffers of one call, freed when it returns
struct Scratch {
  std::vector<void*> bufs;
  cudaError_t err = cudaSuccess;
  template <class T>
  T* alloc(size_t n) {
    void* p = nullptr;
    if (err == cudaSuccess) err = cudaMalloc(&p, sizeof(T) * (n ? n : 1));
    if (err == cudaSuccess) bufs.push_back(p);
    return static_cast<T*>(p);
  }
  template <class T>
  T* upload(const T* h, size_t n, cudaStream_t s) {
    T* d = alloc<T>(n);
    if (err == cudaSuccess && n) err = cudaMemcpyAsync(d, h, sizeof(T) * n, cudaMemcpyHostToDevice, s);
    return d;
  }
  ~Scratch() {
    for (void* p : bufs) cudaFree(p);
  }
};

vh_status ic_err(vh_ctx* ctx, vh_status st, const std::string& msg) {
  ctx->err = msg;
  return st;
}

vh_status ic_cuda(vh_ctx* ctx, cudaError_t e, const char* who) {
  return ic_err(ctx, VH_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
}

vh_status ic_begin(vh_ctx* ctx, const char* who) {
  if (ctx->surf_pending)
    return ic_err(ctx, VH_ERR_STATE, std::string(who) + ": a vh_surface_begin has not ended");
  if (ctx->g.zoff != 0 || ctx->g.nzg != ctx->g.nz)
    return ic_err(ctx, VH_ERR_STATE, std::string(who) + ": the context is a slab of a larger grid");
  const cudaError_t e = cudaSetDevice(ctx->device);
  return e == cudaSuccess ? VH_OK : ic_cuda(ctx, e, who);
}

unsigned blocks(long long n) { return (unsigned)((n + kTpb - 1) / kTpb); }

// Fluid::getZ (src/fld.h:64) of every eta cell
std::vector<double> eta_axis(const vh_ctx* ctx) {
  std::vector<double> eta(ctx->g.nz);
  for (int iz = 0; iz < ctx->g.nz; iz++) eta[iz] = ctx->grid.etamin + iz * ctx->g.dz;
  return eta;
}

// the rapidity constants recomputed per event at 27 GeV
// (src/icGlissando.cpp:188-195, src/icTrento.cpp:243-253)
void rhic27_update(vh_ic_setup& u, int npart) {
  if (u.sNN == 27) {
    const double cent = (double)npart / (2. * 197.);
    u.eta0 = 0.888 - 0.213 * cent;
    u.sigEta = 1.088 - 0.213 * cent;
    u.neta0 = 1.332 - 0.319 * cent;
    u.nsigma = 0.788 - 0.213 * cent;
  }
}

double f_eta(const vh_ic_setup& u, double eta) {
  double fEta = 0.;
  if (std::fabs(eta) < u.eta0)
    fEta = 1.0;
  else if (std::fabs(eta) < u.ybeam)
    fEta = std::exp(-0.5 * std::pow((std::fabs(eta) - u.eta0) / u.sigEta, 2));
  return fEta;
}

double baryon_gauss(const vh_ic_setup& u, double centre_sign_eta) {
  double bg = std::exp(-std::pow(centre_sign_eta, 2) / (2. * u.nsigma * u.nsigma));
  bg /= u.nsigma * std::sqrt(2 * vh::icr::kCPi);
  return bg;
}

// u^eta / u^tau of the setups' shear flow, tanh(A x) sinh(ybeam - |eta|)
// (src/icGlissando.cpp:240-241, src/icTrento.cpp:292-293), [nz][nx]
std::vector<double> shear_vz(const vh_ctx* ctx, const vh_ic_setup& u) {
  const vh::Geo& g = ctx->g;
  const std::vector<double> eta = eta_axis(ctx);
  std::vector<double> vz((size_t)g.nz * g.nx);
  for (int iz = 0; iz < g.nz; iz++)
    for (int ix = 0; ix < g.nx; ix++) {
      const double ueta = std::tanh(u.A * (ctx->grid.xmin + ix * g.dx)) *
                          std::sinh(u.ybeam - std::fabs(eta[iz]));
      const double u0 = std::sqrt(1.0 + ueta * ueta);
      vz[(size_t)iz * g.nx + ix] = ueta / u0;
    }
  return vz;
}

// One normalisation loop of the constructors (src/icGlissando.cpp:164-181,
// src/icTrento.cpp:185-202): norm <- g(sum at norm) norm_old until it moves
// by at most 1e-4; g = (npart sNN / 2 / E)^(3/4) for the entropy, npart / Nb
// for the baryon number.
vh_status norm_loop(vh_ctx* ctx, vh::icr::TermArgs ta, double* d_sum, double* h_sum,
                    double npart, double sNN, bool baryon, double* norm, const char* who) {
  cudaStream_t s = ctx->stream;
  double nrm = 1.0, old;
  int it = 0;
  do {
    old = nrm;
    ta.norm = nrm;
    vh::icr::k_ic_terms<<<blocks(ta.N), kTpb, 0, s>>>(ta);
    vh::icr::k_seq_sum<<<1, vh::icr::kSumThreads, 0, s>>>(ta.terms, ta.N, d_sum);
    cudaError_t e = cudaMemcpyAsync(h_sum, d_sum, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return ic_cuda(ctx, e, who);
    if (baryon)
      nrm = npart / *h_sum * old;
    else
      nrm = std::pow(npart * 0.5 * sNN / *h_sum, 0.75) * old;
    if (++it > vh::icr::kNormMaxIt)
      return ic_err(ctx, VH_ERR_NUMERIC, std::string(who) + ": the normalisation does not converge");
  } while (std::fabs(nrm - old) > 0.0001);
  *norm = nrm;
  return VH_OK;
}

// the end of a call: the s95p convergence flag, errors, the state uploaded
vh_status ic_finish(vh_ctx* ctx, Scratch& sc, const unsigned* d_bad, const char* who) {
  unsigned bad = 0;
  cudaError_t e = sc.err != cudaSuccess ? sc.err : cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ic_cuda(ctx, e, who);
  if (bad) return ic_err(ctx, VH_ERR_NUMERIC, std::string(who) + ": s95p_e did not converge");
  ctx->uploaded = true;
  return VH_OK;
}

vh::icr::ColGeo col_geo(const vh_ctx* ctx) {
  return {ctx->g.nx, ctx->g.ny, ctx->g.nz, ctx->grid.xmin, ctx->grid.ymin, ctx->g.dx, ctx->g.dy};
}

vh::icr::SetArgs set_args(const vh_ctx* ctx, double tau0) {
  vh::icr::SetArgs a{};
  a.nx = ctx->g.nx;
  a.ny = ctx->g.ny;
  a.nz = ctx->g.nz;
  a.N = ctx->g.N;
  a.dx = ctx->g.dx;
  a.dy = ctx->g.dy;
  a.dz = ctx->g.dz;
  a.tau0 = tau0;
  a.E = ctx->eos;
  a.f = ctx->f;
  return a;
}

}  // namespace

extern "C" vh_status vh_ic_setup_named(int model, const char* name, vh_ic_setup* out) {
  if (!name || !out) return VH_ERR_ARG;
  for (const SetupEntry& e : kSetups)
    if (e.model == model && std::strcmp(e.name, name) == 0) {
      *out = e.s;
      return VH_OK;
    }
  return VH_ERR_ARG;
}

extern "C" vh_status vh_init_glissando(vh_ctx* ctx, const vh_glissando_ic* ic, double* norms) {
  static const char* who = "vh_init_glissando";
  if (!ctx || !ic || ic->nevents < 1 || !ic->npart) return VH_ERR_ARG;
  long long nsrc = 0;
  for (int ev = 0; ev < ic->nevents; ev++) {
    if (ic->npart[ev] < 1) return ic_err(ctx, VH_ERR_ARG, std::string(who) + ": an event without sources");
    nsrc += ic->npart[ev];
  }
  if (!ic->x || !ic->y || !ic->c || nsrc > INT32_MAX || !(ic->setup.Rg > 0.))
    return ic_err(ctx, VH_ERR_ARG, std::string(who) + ": sources or Rg missing");
  vh_status st = ic_begin(ctx, who);
  if (st) return st;
  const vh::Geo& g = ctx->g;
  cudaStream_t s = ctx->stream;
  const int nz = g.nz, nev = ic->nevents;
  // per event and eta cell: fEta, the tilt per code sign, the baryon Gaussian
  // (src/icGlissando.cpp:207-221), with the setup's per-event constants
  const std::vector<double> eta = eta_axis(ctx);
  vh_ic_setup u = ic->setup;
  std::vector<double> fEta((size_t)nev * nz), bg((size_t)nev * 2 * nz, 0.), tilt(2 * (size_t)nz);
  std::vector<int> sev((size_t)nsrc);
  for (int iz = 0; iz < nz; iz++)
    for (int sg = 0; sg < 2; sg++) {
      double t = sg == 0 ? 0.5 * (u.etaM + eta[iz]) / u.etaM : 0.5 * (u.etaM - eta[iz]) / u.etaM;
      t = std::max(0.0, t);
      t = std::min(1.0, t);
      tilt[(size_t)sg * nz + iz] = t;
    }
  long long base = 0;
  for (int ev = 0; ev < nev; ev++) {
    rhic27_update(u, ic->npart[ev]);
    for (int iz = 0; iz < nz; iz++) {
      fEta[(size_t)ev * nz + iz] = f_eta(u, eta[iz]);
      if (u.sNN < 100) {
        bg[((size_t)ev * 2 + 0) * nz + iz] = baryon_gauss(u, eta[iz] - u.neta0);
        bg[((size_t)ev * 2 + 1) * nz + iz] = baryon_gauss(u, eta[iz] + u.neta0);
      }
    }
    for (int k = 0; k < ic->npart[ev]; k++) sev[(size_t)(base + k)] = ev;
    base += ic->npart[ev];
  }
  std::vector<double> cosh_eta(nz);
  for (int iz = 0; iz < nz; iz++) cosh_eta[iz] = std::cosh(eta[iz]);
  const std::vector<double> vz = shear_vz(ctx, ic->setup);
  const bool baryon = ic->setup.sNN < 100;

  Scratch sc;
  vh::icr::GlissArgs a{};
  a.g = col_geo(ctx);
  a.ns = (int)(3.0 * ic->setup.Rg / g.dx);
  a.Rg = ic->setup.Rg;
  a.alphaMix = ic->setup.alphaMix;
  a.baryon = baryon;
  a.nsrc = (int)nsrc;
  a.sx = sc.upload(ic->x, (size_t)nsrc, s);
  a.sy = sc.upload(ic->y, (size_t)nsrc, s);
  a.sc = sc.upload(ic->c, (size_t)nsrc, s);
  a.sev = sc.upload(sev.data(), sev.size(), s);
  a.fEta = sc.upload(fEta.data(), fEta.size(), s);
  a.tilt = sc.upload(tilt.data(), tilt.size(), s);
  a.bg = sc.upload(bg.data(), bg.size(), s);
  a.rho = sc.alloc<double>(g.N);
  a.nrho = sc.alloc<double>(g.N);
  double* terms = sc.alloc<double>(g.N);
  const double* d_cosh = sc.upload(cosh_eta.data(), cosh_eta.size(), s);
  const double* d_vz = sc.upload(vz.data(), vz.size(), s);
  double* d_sum = sc.alloc<double>(1);
  unsigned* d_bad = sc.alloc<unsigned>(1);
  if (sc.err == cudaSuccess) sc.err = cudaMemsetAsync(d_bad, 0, sizeof(unsigned), s);
  if (sc.err != cudaSuccess) return ic_cuda(ctx, sc.err, who);
  const long long ncol = (long long)g.nx * g.ny;
  const long long nch = (nz + vh::icr::kKz - 1) / vh::icr::kKz;
  vh::icr::k_gliss_rho<<<blocks(ncol * nch), kTpb, 0, s>>>(a);

  // sNorm, nNorm (src/icGlissando.cpp:164-181) against np_tot / nevents
  double h_sum = 0.;
  const double npart = (double)(nsrc / nev);
  vh::icr::TermArgs ta{g.nx, g.ny, nz, g.N, g.dx, g.dy, g.dz, ctx->tau,
                       vh::icr::TERM_E_DXDY, 1.0, (double)nev, a.rho, d_cosh, terms, d_bad};
  double sNorm = 1.0, nNorm = 0.0;
  if ((st = norm_loop(ctx, ta, d_sum, &h_sum, npart, ic->setup.sNN, false, &sNorm, who))) return st;
  if (baryon) {
    ta.mode = vh::icr::TERM_NB;
    ta.rho = a.nrho;
    if ((st = norm_loop(ctx, ta, d_sum, &h_sum, npart, ic->setup.sNN, true, &nNorm, who))) return st;
  }
  vh::icr::SetArgs sa = set_args(ctx, ctx->tau);
  sa.sdiv = 1;
  sa.baryon = baryon;
  sa.sNorm = sNorm;
  sa.nNorm = nNorm;
  sa.nev = nev;
  sa.rho = a.rho;
  sa.nrho = a.nrho;
  sa.vz = d_vz;
  sa.bad = d_bad;
  vh::icr::k_ic_set<<<blocks(g.N), kTpb, 0, s>>>(sa);
  if ((st = ic_finish(ctx, sc, d_bad, who))) return st;
  if (norms) {
    norms[0] = sNorm;
    norms[1] = nNorm;
  }
  return VH_OK;
}

extern "C" vh_status vh_init_trento(vh_ctx* ctx, const vh_trento_ic* ic, double* norms) {
  static const char* who = "vh_init_trento";
  if (!ctx || !ic || ic->nevents < 1 || !ic->ngrid || !ic->gmax || !ic->npart || !ic->grid)
    return VH_ERR_ARG;
  const int nev = ic->nevents;
  std::vector<long long> goff(nev);
  long long nval = 0;
  for (int ev = 0; ev < nev; ev++) {
    if (ic->ngrid[ev] < 2 || !(ic->gmax[ev] > 0.))
      return ic_err(ctx, VH_ERR_ARG, std::string(who) + ": need grid-nsteps >= 2 and grid-max > 0");
    goff[ev] = nval;
    nval += (long long)ic->ngrid[ev] * ic->ngrid[ev];
  }
  vh_status st = ic_begin(ctx, who);
  if (st) return st;
  const vh::Geo& g = ctx->g;
  cudaStream_t s = ctx->stream;
  const int nz = g.nz;
  // per event and eta cell: fEta and the baryon Gaussian of eta's sign
  // (src/icTrento.cpp:262-273)
  const std::vector<double> eta = eta_axis(ctx);
  vh_ic_setup u = ic->setup;
  std::vector<double> fEta((size_t)nev * nz), bgz((size_t)nev * nz, 0.);
  for (int ev = 0; ev < nev; ev++) {
    rhic27_update(u, ic->npart[ev]);
    for (int iz = 0; iz < nz; iz++) {
      fEta[(size_t)ev * nz + iz] = f_eta(u, eta[iz]);
      if (u.sNN < 100)
        bgz[(size_t)ev * nz + iz] =
            baryon_gauss(u, eta[iz] > 0 ? eta[iz] - u.neta0 : eta[iz] + u.neta0);
    }
  }
  std::vector<double> cosh_eta(nz);
  for (int iz = 0; iz < nz; iz++) cosh_eta[iz] = std::cosh(eta[iz]);
  const std::vector<double> vz = shear_vz(ctx, ic->setup);
  const bool baryon = ic->setup.sNN < 100;

  Scratch sc;
  vh::icr::TrentoArgs a{};
  a.g = col_geo(ctx);
  a.baryon = baryon;
  a.nev = nev;
  a.grid = sc.upload(ic->grid, (size_t)nval, s);
  a.goff = sc.upload(goff.data(), goff.size(), s);
  a.gn = sc.upload(ic->ngrid, (size_t)nev, s);
  a.gmax = sc.upload(ic->gmax, (size_t)nev, s);
  a.fEta = sc.upload(fEta.data(), fEta.size(), s);
  a.bgz = sc.upload(bgz.data(), bgz.size(), s);
  a.rho = sc.alloc<double>(g.N);
  a.nrho = sc.alloc<double>(g.N);
  double* terms = sc.alloc<double>(g.N);
  const double* d_cosh = sc.upload(cosh_eta.data(), cosh_eta.size(), s);
  const double* d_vz = sc.upload(vz.data(), vz.size(), s);
  double* d_sum = sc.alloc<double>(1);
  unsigned* d_bad = sc.alloc<unsigned>(1);
  if (sc.err == cudaSuccess) sc.err = cudaMemsetAsync(d_bad, 0, sizeof(unsigned), s);
  if (sc.err != cudaSuccess) return ic_cuda(ctx, sc.err, who);
  const long long ncol = (long long)g.nx * g.ny;
  const long long nch = (nz + vh::icr::kKz - 1) / vh::icr::kKz;
  vh::icr::k_trento_rho<<<blocks(ncol * nch), kTpb, 0, s>>>(a);

  // below 2760 GeV, sNorm (and below 100 GeV nNorm) against the last
  // event's npart (src/icTrento.cpp:183-206); else sNorm = 1
  double h_sum = 0., sNorm = 1.0, nNorm = 0.0;
  const double npart = (double)ic->npart[nev - 1];
  if (ic->setup.sNN < 2760) {
    vh::icr::TermArgs ta{g.nx, g.ny, nz, g.N, g.dx, g.dy, g.dz, ctx->tau,
                         vh::icr::TERM_E, 1.0, (double)nev, a.rho, d_cosh, terms, d_bad};
    if ((st = norm_loop(ctx, ta, d_sum, &h_sum, npart, ic->setup.sNN, false, &sNorm, who)))
      return st;
    if (baryon) {
      ta.mode = vh::icr::TERM_NB;
      ta.rho = a.nrho;
      if ((st = norm_loop(ctx, ta, d_sum, &h_sum, npart, ic->setup.sNN, true, &nNorm, who)))
        return st;
    }
  }
  vh::icr::SetArgs sa = set_args(ctx, ctx->tau);
  sa.sdiv = 0;
  sa.baryon = baryon;
  sa.sNorm = sNorm;
  sa.nNorm = nNorm;
  sa.nev = nev;
  sa.rho = a.rho;
  sa.nrho = a.nrho;
  sa.vz = d_vz;
  sa.bad = d_bad;
  vh::icr::k_ic_set<<<blocks(g.N), kTpb, 0, s>>>(sa);
  if ((st = ic_finish(ctx, sc, d_bad, who))) return st;
  if (norms) {
    norms[0] = sNorm;
    norms[1] = nNorm;
  }
  return VH_OK;
}

extern "C" vh_status vh_init_gubser(vh_ctx* ctx) {
  static const char* who = "vh_init_gubser";
  if (!ctx) return VH_ERR_ARG;
  vh_status st = ic_begin(ctx, who);
  if (st) return st;
  Scratch sc;
  unsigned* d_bad = sc.alloc<unsigned>(1);
  if (sc.err == cudaSuccess) sc.err = cudaMemsetAsync(d_bad, 0, sizeof(unsigned), ctx->stream);
  if (sc.err != cudaSuccess) return ic_cuda(ctx, sc.err, who);
  vh::icr::k_ic_gubser<<<blocks(ctx->g.N), kTpb, 0, ctx->stream>>>(
      ctx->g, ctx->grid.xmin, ctx->grid.ymin, ctx->tau, ctx->eos, ctx->f);
  return ic_finish(ctx, sc, d_bad, who);
}

extern "C" vh_status vh_init_table(vh_ctx* ctx, const vh_table_ic* ic) {
  static const char* who = "vh_init_table";
  if (!ctx || !ic || !ic->x || !ic->y || !ic->val) return VH_ERR_ARG;
  if (ic->nx < 2 || ic->ny < 2)
    return ic_err(ctx, VH_ERR_ARG, std::string(who) + ": the table needs 2 x 2 points at least");
  vh_status st = ic_begin(ctx, who);
  if (st) return st;
  const vh::Geo& g = ctx->g;
  cudaStream_t s = ctx->stream;
  // the rapidity factor of IC::setIC, src/ic.cpp:33-35
  const std::vector<double> eta = eta_axis(ctx);
  std::vector<double> etaF(g.nz);
  for (int iz = 0; iz < g.nz; iz++) {
    const double eta1 = std::fabs(eta[iz]) < 1.3 ? 0.0 : std::fabs(eta[iz]) - 1.3;
    etaF[iz] = std::exp(-eta1 * eta1 / 2.1 / 2.1) * (std::fabs(eta[iz]) < 5.3 ? 1.0 : 0.0);
  }
  const long long nt = (long long)ic->nx * ic->ny;
  Scratch sc;
  const double* d_val = sc.upload(ic->val, (size_t)nt, s);
  double* d_t = sc.alloc<double>((size_t)nt);
  const double* d_etaF = sc.upload(etaF.data(), etaF.size(), s);
  unsigned* d_bad = sc.alloc<unsigned>(1);
  if (sc.err == cudaSuccess) sc.err = cudaMemsetAsync(d_bad, 0, sizeof(unsigned), s);
  if (sc.err != cudaSuccess) return ic_cuda(ctx, sc.err, who);
  vh::icr::k_table_prep<<<blocks(nt), kTpb, 0, s>>>(d_val, nt, ic->factor, ic->glauber_var, d_t,
                                                    d_bad);
  vh::icr::TableArgs a{};
  a.g = g;
  a.xmin = ctx->grid.xmin;
  a.ymin = ctx->grid.ymin;
  a.tau = ctx->tau;
  a.NX = ic->nx;
  a.NY = ic->ny;
  a.txmin = ic->x[0];
  a.txmax = ic->x[ic->nx - 1];
  a.tymin = ic->y[0];
  a.tymax = ic->y[ic->ny - 1];
  a.t = d_t;
  a.etaF = d_etaF;
  a.E = ctx->eos;
  a.f = ctx->f;
  vh::icr::k_ic_table<<<blocks(g.N), kTpb, 0, s>>>(a);
  return ic_finish(ctx, sc, d_bad, who);
}

extern "C" vh_status vh_init_urqmd(vh_ctx* ctx, const vh_urqmd_ic* ic) {
  static const char* who = "vh_init_urqmd";
  if (!ctx || !ic || ic->nevents < 1 || !ic->npart || !ic->p || !ic->id || !ic->charge)
    return VH_ERR_ARG;
  long long n = 0;
  for (int ev = 0; ev < ic->nevents; ev++) {
    if (ic->npart[ev] < 1) return ic_err(ctx, VH_ERR_ARG, std::string(who) + ": an event without particles");
    n += ic->npart[ev];
  }
  if (n > INT32_MAX / 64 || !(ic->Rgt > 0.) || !(ic->Rgz >= 0.))
    return ic_err(ctx, VH_ERR_ARG, std::string(who) + ": need Rgt > 0, Rgz >= 0");
  vh_status st = ic_begin(ctx, who);
  if (st) return st;
  const vh::Geo& g = ctx->g;
  cudaStream_t s = ctx->stream;
  vh::icr::UrqmdArgs a{};
  a.g = g;
  a.xmin = ctx->grid.xmin;
  a.ymin = ctx->grid.ymin;
  a.zmin = ctx->grid.etamin;
  a.tau0 = ctx->tau;
  a.Rgx = a.Rgy = ic->Rgt;
  a.Rgz = ic->Rgz;
  a.nev = ic->nevents;
  // the stencil half-widths (src/icPartUrqmd.cpp:36-38)
  a.nsx = (int)(6.0 * a.Rgx / g.dx);
  a.nsy = (int)(6.0 * a.Rgy / g.dy);
  a.nsz = (int)(1.5 * a.Rgz / g.dz);
  a.n = (int)n;
  const int nzs = 2 * a.nsz + 1;
  // per particle: the stencil centre (rounded as the module rounds), gamma_z
  // and the cosh / sinh of every stencil plane's rapidity offset, with the C
  // library; the tiles each stencil meets, in particle order
  std::vector<int> c3(3 * (size_t)n);
  std::vector<double> gz(n), csh((size_t)n * nzs * 2);
  a.ntx = (g.nx + vh::icr::kUqTx - 1) / vh::icr::kUqTx;
  const int nty = (g.ny + vh::icr::kUqTy - 1) / vh::icr::kUqTy;
  std::vector<std::vector<int>> tiles((size_t)a.ntx * nty);
  for (long long ip = 0; ip < n; ip++) {
    const double* q = ic->p + 8 * ip;
    const int ixc = (int)std::round((q[1] - a.xmin) / g.dx);
    const int iyc = (int)std::round((q[2] - a.ymin) / g.dy);
    const int izc = (int)std::round((q[3] - a.zmin) / g.dz);
    c3[3 * ip] = ixc;
    c3[3 * ip + 1] = iyc;
    c3[3 * ip + 2] = izc;
    gz[ip] = std::cosh(q[7] - q[3]);
    for (int k = 0; k < nzs; k++) {
      const int iz = izc - a.nsz + k;
      const double zdiff = q[3] - (a.zmin + iz * g.dz);
      csh[((size_t)ip * nzs + k) * 2] = std::cosh(q[7] - q[3] + zdiff);
      csh[((size_t)ip * nzs + k) * 2 + 1] = std::sinh(q[7] - q[3] + zdiff);
    }
    const int x0 = std::max(1, ixc - a.nsx), x1 = std::min(g.nx - 1, ixc + a.nsx);
    const int y0 = std::max(1, iyc - a.nsy), y1 = std::min(g.ny - 1, iyc + a.nsy);
    const int z0 = std::max(1, izc - a.nsz), z1 = std::min(g.nz - 1, izc + a.nsz);
    if (x0 > x1 || y0 > y1 || z0 > z1) continue;  // the stencil misses the grid
    for (int ty = y0 / vh::icr::kUqTy; ty <= y1 / vh::icr::kUqTy; ty++)
      for (int tx = x0 / vh::icr::kUqTx; tx <= x1 / vh::icr::kUqTx; tx++)
        tiles[(size_t)ty * a.ntx + tx].push_back((int)ip);
  }
  size_t nlist = 0;
  for (const std::vector<int>& t : tiles) nlist += t.size();
  if (nlist > (size_t)INT32_MAX)
    return ic_err(ctx, VH_ERR_ARG, std::string(who) + ": too many particle-tile pairs");
  std::vector<int> toff(tiles.size() + 1, 0), tlist;
  tlist.reserve(nlist);
  for (size_t t = 0; t < tiles.size(); t++) {
    toff[t + 1] = toff[t] + (int)tiles[t].size();
    tlist.insert(tlist.end(), tiles[t].begin(), tiles[t].end());
  }
  Scratch sc;
  a.p = sc.upload(ic->p, 8 * (size_t)n, s);
  a.id = sc.upload(ic->id, (size_t)n, s);
  a.charge = sc.upload(ic->charge, (size_t)n, s);
  a.c3 = sc.upload(c3.data(), c3.size(), s);
  a.gz = sc.upload(gz.data(), gz.size(), s);
  a.csh = sc.upload(csh.data(), csh.size(), s);
  a.norm = sc.alloc<double>((size_t)n);
  a.toff = sc.upload(toff.data(), toff.size(), s);
  a.tlist = sc.upload(tlist.data(), tlist.size(), s);
  a.T = sc.alloc<double>(6 * (size_t)g.N);
  unsigned* d_bad = sc.alloc<unsigned>(1);
  if (sc.err == cudaSuccess) sc.err = cudaMemsetAsync(d_bad, 0, sizeof(unsigned), s);
  if (sc.err != cudaSuccess) return ic_cuda(ctx, sc.err, who);
  vh::icr::k_urqmd_norm<<<blocks(n), kTpb, 0, s>>>(a);
  vh::icr::k_urqmd_T<<<dim3((unsigned)tiles.size(), (unsigned)g.nz), vh::icr::kUqTx * vh::icr::kUqTy,
                       0, s>>>(a);
  // the module's transformPV: the reference's Newton at its own tolerance,
  // whatever the context's steps use
  vh::EosDev E = ctx->eos;
  E.tol = 0.00001;
  E.slope = 0;
  E.vguess = nullptr;
  E.stats = nullptr;
  vh::icr::k_urqmd_set<<<blocks(g.N), kTpb, 0, s>>>(a, E, ctx->f);
  return ic_finish(ctx, sc, d_bad, who);
}
