// vh_step.cu -- the kernels of one hydro timestep (Hydro::performStep,
// src/hdo.cpp:1016-1134) on a structure-of-arrays FP64 grid.
//
// Data-parallel restructuring of the reference's sequential loops:
//  * face kernels compute each HLLE face flux once (two con2prims per face)
//    into a per-direction face array; a cell kernel then gathers the six
//    faces in the reference's accumulation order (x-, x+, y-, y+, z-, z+,
//    source), which keeps every cell's FP64 sum identical to the reference;
//  * the viscous part stores the two cell-centred con2prims that every
//    viscous stage re-derives (Qh at tau_n + dt/2 and Qh at tau_{n+1}) once
//    per cell and reuses them, which is exact because the reference
//    recomputes them from identical inputs;
//  * ghost cells are a gather from a per-dimension source map simulated on
//    the host from the reference's copy sequence (z, then y, then x).
#include <cuda_runtime.h>

#include <algorithm>

#include "vh_physics.cuh"
#include "vh_step.cuh"

namespace vh {

// -------------------------------------------------------------- updateM
// Fluid::updateM, src/fld.cpp:384-423 (both passes; out of place).
__device__ __forceinline__ void d_update_m(const Geo& g, const double* __restrict__ m,
                                           double* __restrict__ mo, const double* __restrict__ clk,
                                           long long blk) {
  const double tau = clk[0], dt = clk[1];  // the step's clock (device)
  const long long i = blk * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  const long long N = g.N;
  double d0 = 0., d1 = 0., d2 = 0.;
  if (maxM(m, N, i) < 1.) {
    if (m[cidx(g, ix + 1, iy, iz)] >= 1. || m[cidx(g, ix - 1, iy, iz)] >= 1.) d0 = dt / g.dx;
    if (m[N + cidx(g, ix, iy + 1, iz)] >= 1. || m[N + cidx(g, ix, iy - 1, iz)] >= 1.)
      d1 = dt / g.dy;
    if (m[2 * N + cidx(g, ix, iy, iz + 1)] >= 1. || m[2 * N + cidx(g, ix, iy, iz - 1)] >= 1.)
      d2 = dt / g.dz / tau;
    if (d0 == 0. && d1 == 0.) {
      if (maxM(m, N, cidx(g, ix + 1, iy + 1, iz)) >= 1. ||
          maxM(m, N, cidx(g, ix + 1, iy - 1, iz)) >= 1. ||
          maxM(m, N, cidx(g, ix - 1, iy + 1, iz)) >= 1. ||
          maxM(m, N, cidx(g, ix - 1, iy - 1, iz)) >= 1.) {
        d0 = 0.707 * dt / g.dx;
        d1 = 0.707 * dt / g.dy;
      }
    }
  }
  // Cell::addM, src/cll.h:147-151, for X, Y, Z in turn
  double a0 = m[i], a1 = m[N + i], a2 = m[2 * N + i];
  a0 += d0;
  if (a0 > 0.9) a0 = a1 = a2 = 1.;
  a1 += d1;
  if (a1 > 0.9) a0 = a1 = a2 = 1.;
  a2 += d2;
  if (a2 > 0.9) a0 = a1 = a2 = 1.;
  mo[i] = a0;
  mo[N + i] = a1;
  mo[2 * N + i] = a2;
}
__global__ void k_update_m(Geo g, const double* __restrict__ m, double* __restrict__ mo,
                           const double* __restrict__ clk) {
  d_update_m(g, m, mo, clk, blockIdx.x);
}


// ------------------------------------------------------------ face flux
// One HLLE face between cell i and its +DIR neighbour (Hydro::hlle_flux with
// Cell::getPrimVarRight / getPrimVarLeft or their H variants,
// src/cll.cpp:106-204).  F[c*N + i] holds the flux of the face on the +DIR
// side of cell i (0 where the reference adds nothing).
// Occupancy (measured over 100 steps of the 101x101x51 event): 8 blocks of
// 128 threads per SM (64 registers, a few spills) are 11 % faster than the
// unbounded build (80 registers, 6 blocks); 10 blocks are slower.  The
// same sweep set k_update to 12 blocks (-14 %), k_visc_prims to 8 (-14 %),
// k_visc_update to 8 (-10 %); k_is_advect stays unbounded (8 blocks: +52 %).
template <int DIR, bool PRED, int EK>
// 7 blocks of 128 per SM (72 registers): measured against 6 and 8 blocks on
// the 300-step event, 3 % faster than 8 (64 registers, more spills)
__device__ __forceinline__ void d_face(const Geo& g, const EosDev& E,
                                       const double* __restrict__ QQ,
                                       const double* __restrict__ m, double* __restrict__ F,
                                       const double* __restrict__ clk, unsigned* err,
                                       long long blk) {
  const double tau = clk[0], dt = clk[1];  // the step's clock (device)
  const long long i = blk * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  const long long N = g.N;
  long long L = i, Lm, R, Rp;
  if (DIR == X_) {
    if (ix >= g.nx - 1) return;
    Lm = cidx(g, ix - 1, iy, iz);
    R = cidx(g, ix + 1, iy, iz);
    Rp = cidx(g, ix + 2, iy, iz);
  } else if (DIR == Y_) {
    if (iy >= g.ny - 1) return;
    Lm = cidx(g, ix, iy - 1, iz);
    R = cidx(g, ix, iy + 1, iz);
    Rp = cidx(g, ix, iy + 2, iz);
  } else {
    if (iz >= g.nz - 1) return;
    Lm = cidx(g, ix, iy, iz - 1);
    R = cidx(g, ix, iy, iz + 1);
    Rp = cidx(g, ix, iy, iz + 2);
  }
  double qlr[14];  // the two reconstructed states, then divided by tau as one batch
#pragma unroll
  for (int k = 0; k < 7; k++) {
    const double a = QQ[k * N + Lm], b = QQ[k * N + L], c = QQ[k * N + R], d = QQ[k * N + Rp];
    const double dQl = minmod((c - b) / 2., (b - a) / 2.);
    qlr[k] = b + dQl;
    const double dQr = minmod((d - c) / 2., (c - b) / 2.);
    qlr[7 + k] = c - dQr;
  }
  div_batch<14>(qlr, tau, 1.0 / tau, crm::mk_den_ok(tau));
  double ql[7], qr[7];
#pragma unroll
  for (int k = 0; k < 7; k++) {
    ql[k] = qlr[k];
    qr[k] = qlr[7 + k];
  }
  Prim pl, pr;
  transform_pv<EK>(E, ql, pl, c2p_guess(E, L));
  transform_pv<EK>(E, qr, pr, c2p_guess(E, R));
  const double dxdir = DIR == X_ ? g.dx : (DIR == Y_ ? g.dy : g.dz);
  double fl[7];
  unsigned e = 0;
  const bool ok = hlle_face(DIR, PRED, tau, dt, dxdir, pl, pr, m[(DIR - 1) * N + L],
                            m[(DIR - 1) * N + R], fl, e);
  if (e) atomicOr(err, e);
#pragma unroll
  for (int k = 0; k < 7; k++) F[k * N + i] = ok ? fl[k] : 0.;
}
template <int DIR, bool PRED, int EK>
__global__ void __launch_bounds__(128, 7) k_face(Geo g, EosDev E, const double* __restrict__ QQ,
                                              const double* __restrict__ m,
                                              double* __restrict__ F, const double* __restrict__ clk,
                                              unsigned* err) {
  d_face<DIR, PRED, EK>(g, E, QQ, m, F, clk, err, blockIdx.x);
}


// --------------------------------------------------- ideal cell update
// Gathers the six face fluxes and the Milne source (Hydro::source_step,
// src/hdo.cpp:307-353), then Cell::updateQtoQhByFlux (predictor) or
// Cell::updateByFlux (corrector), src/cll.cpp:70-88.
template <bool PRED, int EK>
__device__ __forceinline__ void d_update(const Geo& g, const EosDev& E, double* __restrict__ Q,
                                         double* __restrict__ Qh, double* __restrict__ Qprev,
                                         const double* __restrict__ Fx,
                                         const double* __restrict__ Fy,
                                         const double* __restrict__ Fz,
                                         const double* __restrict__ clk, unsigned* err,
                                         double* __restrict__ pB, double* __restrict__ pA,
                                         long long blk) {
  const double tau = clk[0], dt = clk[1];  // the step's clock (device)
  const long long i = blk * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  const long long N = g.N;
  const long long sy = g.nx, sz = (long long)g.nx * g.ny;
  double fl[7];
#pragma unroll
  for (int k = 0; k < 7; k++) {
    double a = 0.;
    if (ix > 0) a += Fx[k * N + i - 1];
    if (ix < g.nx - 1) a += -Fx[k * N + i];
    if (iy > 0) a += Fy[k * N + i - sy];
    if (iy < g.ny - 1) a += -Fy[k * N + i - 0];
    if (iz > 0) a += Fz[k * N + i - sz];
    if (iz < g.nz - 1) a += -Fz[k * N + i];
    fl[k] = a;
  }
  const double* field = PRED ? Q : Qh;
  const double tau1 = PRED ? tau : tau + 0.5 * dt;
  const double _dt = PRED ? dt / 2. : dt;
  double q[7], qin[7];
#pragma unroll
  for (int k = 0; k < 7; k++) qin[k] = field[k * N + i];
  q_over(qin, tau1, q);
  Prim pp;
  transform_pv<EK>(E, q, pp, c2p_guess(E, i));
  if (!PRED && pA) {
    // con2prim(Qh / (tau_n + dt/2)) is the viscous stage's A =
    // con2prim(Qh / (tau_{n+1} - dt/2)) for every cell that the ghost copy
    // does not overwrite, whenever the divisors agree bit for bit
    pA[0 * N + i] = pp.e;
    pA[1 * N + i] = pp.p;
    pA[2 * N + i] = pp.nb;
    pA[3 * N + i] = pp.nq;
    pA[4 * N + i] = pp.ns;
    pA[5 * N + i] = pp.vx;
    pA[6 * N + i] = pp.vy;
    pA[7 * N + i] = pp.vz;
  }
  if (PRED && pB) {
    // con2prim(Q_n / tau_n) is the viscous stage's B = con2prim(Qprev /
    // (tau_{n+1} - dt)) whenever (tau_n + dt) - dt == tau_n: kept for it
    // as its four-velocity and e (the same arithmetic as k_visc_prims)
    const double ut = 1.0 / sqrt(1.0 - pp.vx * pp.vx - pp.vy * pp.vy - pp.vz * pp.vz);
    pB[0 * N + i] = ut;
    pB[1 * N + i] = ut * pp.vx;
    pB[2 * N + i] = ut * pp.vy;
    pB[3 * N + i] = ut * pp.vz;
    pB[4 * N + i] = pp.e;
  }
  double kk[7];
  kk[T_] = -q[T_] * pp.vz * pp.vz - pp.p * (1. + pp.vz * pp.vz);
  kk[X_] = 0.;
  kk[Y_] = 0.;
  kk[Z_] = -q[Z_];
  kk[NB_] = 0.;
  kk[NQ_] = 0.;
  kk[NS_] = 0.;
#pragma unroll
  for (int k = 0; k < 7; k++) kk[k] *= _dt;
  if (kk[NB_] != kk[NB_]) {
    atomicOr(err, (unsigned)ERR_SOURCE_NAN);
  } else {
#pragma unroll
    for (int k = 0; k < 7; k++) fl[k] += kk[k];
  }
  if (PRED) {
#pragma unroll
    for (int k = 0; k < 7; k++) {
      const double qk = Q[k * N + i];
      Qprev[k * N + i] = qk;
      Qh[k * N + i] = qk + fl[k];
    }
  } else {
    if (!(Q[i] + fl[0] < 0.)) {
#pragma unroll
      for (int k = 0; k < 7; k++) Q[k * N + i] += fl[k];
    }
  }
}
template <bool PRED, int EK>
__global__ void __launch_bounds__(128, 12) k_update(Geo g, EosDev E, double* __restrict__ Q,
                                                double* __restrict__ Qh,
                                                double* __restrict__ Qprev,
                                                const double* __restrict__ Fx,
                                                const double* __restrict__ Fy,
                                                const double* __restrict__ Fz, const double* __restrict__ clk, unsigned* err,
                                                double* __restrict__ pB, double* __restrict__ pA) {
  d_update<PRED, EK>(g, E, Q, Qh, Qprev, Fx, Fy, Fz, clk, err, pB, pA, blockIdx.x);
}


// ------------------------------------------------------------- ghosts
// Fluid::correctImagCells (FULL = false: Q and Qh) and correctImagCellsFull
// (FULL = true: Q, pi, Pi), src/fld.cpp:211-382, as a gather from the
// per-dimension source maps; copies into a ghost zero the row when Q_t < 0
// (Cell::setQ / setQh).
template <bool FULL>
__device__ __forceinline__ void d_ghost(const Geo& g, const int* __restrict__ src,
                                        const unsigned char* __restrict__ isdst,
                                        double* __restrict__ Q, double* __restrict__ Qh,
                                        double* __restrict__ pi, double* __restrict__ Pi,
                                        long long blk) {
  const long long i = blk * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  const int* sx = src;
  const int* sy = src + g.nx;
  const int* sz = src + g.nx + g.ny;
  if (!(isdst[ix] | isdst[g.nx + iy] | isdst[g.nx + g.ny + iz])) return;
  const long long N = g.N;
  const long long s = (long long)sx[ix] + (long long)g.nx * (sy[iy] + (long long)g.ny * sz[iz]);
  {
    double q[7];
#pragma unroll
    for (int k = 0; k < 7; k++) q[k] = Q[k * N + s];
    const bool neg = q[0] < 0.;
#pragma unroll
    for (int k = 0; k < 7; k++) Q[k * N + i] = neg ? 0. : q[k];
  }
  if (!FULL) {
    double q[7];
#pragma unroll
    for (int k = 0; k < 7; k++) q[k] = Qh[k * N + s];
    const bool neg = q[0] < 0.;
#pragma unroll
    for (int k = 0; k < 7; k++) Qh[k * N + i] = neg ? 0. : q[k];
  } else {
    double p[10];
#pragma unroll
    for (int k = 0; k < 10; k++) p[k] = pi[k * N + s];
    const double P = Pi[s];
#pragma unroll
    for (int k = 0; k < 10; k++) pi[k * N + i] = p[k];
    Pi[i] = P;
  }
}
template <bool FULL>
__global__ void k_ghost(Geo g, const int* __restrict__ src, const unsigned char* __restrict__ isdst,
                        double* __restrict__ Q, double* __restrict__ Qh,
                        double* __restrict__ pi, double* __restrict__ Pi) {
  d_ghost<FULL>(g, src, isdst, Q, Qh, pi, Pi, blockIdx.x);
}


// ------------------------------------------------ viscous cell prims
// Per-cell inputs of the viscous stages, one thread per cell:
//  A  = con2prim(Qh / (tau - dt/2))  (getPrimVarHCenter in ISformal, NSquant,
//                                     visc_flux, visc_source_step),
//  D  = con2prim(Qh / tau)           (the six NSquant neighbour velocities),
//  thermodynamics at A: T, muB, p, s, eta/s, zeta/s, tau_pi, tau_Pi, 9/70/p
//                                    (src/hdo.cpp:427-432, 727-749),
//  B  = con2prim(Qprev / (tau - dt)), C = con2prim(Q / tau) as four-velocities
//                                    (NSquant's time derivative,
//                                     src/hdo.cpp:419-446), only where
//                                     NSquant reaches them (matter, no vacuum
//                                     neighbour).
__device__ __forceinline__ double maxM_at(const Geo& g, const double* __restrict__ m, int ix,
                                          int iy, int iz);

template <int EK>
__device__ __forceinline__ void d_visc_prims(const Geo& g, const EosDev& E, const TrDev& tr,
                                             const double* __restrict__ Q,
                                             const double* __restrict__ Qprev,
                                             const double* __restrict__ Qh,
                                             const double* __restrict__ m, double* __restrict__ pA,
                                             double* __restrict__ pD, double* __restrict__ pTh,
                                             double* __restrict__ pBC,
                                             const double* __restrict__ clk,
                                             const unsigned char* __restrict__ isdst,
                                             long long blk) {
  const double dt = clk[1], tau = clk[0] + dt;  // tau_{n+1} (src/hdo.cpp:1095)
  const long long i = blk * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const long long N = g.N;
  double q[7], qh[7];
#pragma unroll
  for (int k = 0; k < 7; k++) qh[k] = Qh[k * N + i];
  const double tA = tau - dt / 2.;
  Prim a;
  int gx, gy, gz;
  coords(g, i, gx, gy, gz);
  // A is the corrector's con2prim (k_update<false> stored it in pA) when
  // its divisor tau_n + dt/2 equals tA bit for bit and the ghost copy has
  // not changed this cell's Qh since
  if (tA == clk[0] + 0.5 * dt && !(isdst[gx] | isdst[g.nx + gy] | isdst[g.nx + g.ny + gz])) {
    a.e = pA[0 * N + i];
    a.p = pA[1 * N + i];
    a.nb = pA[2 * N + i];
    a.nq = pA[3 * N + i];
    a.ns = pA[4 * N + i];
    a.vx = pA[5 * N + i];
    a.vy = pA[6 * N + i];
    a.vz = pA[7 * N + i];
  } else {
    q_over(qh, tA, q);
    transform_pv<EK>(E, q, a, c2p_guess(E, i));
    pA[0 * N + i] = a.e;
    pA[1 * N + i] = a.p;
    pA[2 * N + i] = a.nb;
    pA[3 * N + i] = a.nq;
    pA[4 * N + i] = a.ns;
    pA[5 * N + i] = a.vx;
    pA[6 * N + i] = a.vy;
    pA[7 * N + i] = a.vz;
  }
  q_over(qh, tau, q);
  Prim d;
  transform_pv<EK>(E, q, d, c2p_guess(E, i));
  pD[0 * N + i] = d.e;
  pD[1 * N + i] = d.vx;
  pD[2 * N + i] = d.vy;
  pD[3 * N + i] = d.vz;
  if (a.e <= 0.) return;
  {
    double T, mub, mus, p;
    eos_eval<EK>(E, a.e, a.nb, T, mub, mus, p);
    // EoS::s at the same point (eos_s, muq = 0) from this lookup
    const double s = T > 0.0 ? ddivp(a.e + p - mub * a.nb - 0. * a.nq - mus * a.ns, T) : 0.;
    const double etaS = tr_etaS(tr, a.e, a.nb, T, mub, s, p);
    const double zetaS = tr_zetaS(tr, a.e, T, s, p);
    double taupi, tauPi;
    tr_getTau_from(a.e, T, s, p, etaS, zetaS, taupi, tauPi);
    pTh[0 * N + i] = T;
    pTh[1 * N + i] = mub;
    pTh[2 * N + i] = p;
    pTh[3 * N + i] = s;
    pTh[4 * N + i] = etaS;
    pTh[5 * N + i] = zetaS;
    pTh[6 * N + i] = taupi;
    pTh[7 * N + i] = tauPi;
    pTh[8 * N + i] = 9. / 70. / p;  // eos_p at the same point is this p
  }
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  const bool vac = maxM_at(g, m, ix + 1, iy, iz) <= 0.9 || maxM_at(g, m, ix, iy + 1, iz) <= 0.9 ||
                   maxM_at(g, m, ix - 1, iy, iz) <= 0.9 || maxM_at(g, m, ix, iy - 1, iz) <= 0.9 ||
                   maxM_at(g, m, ix + 1, iy + 1, iz) <= 0.9 ||
                   maxM_at(g, m, ix + 1, iy - 1, iz) <= 0.9 ||
                   maxM_at(g, m, ix - 1, iy + 1, iz) <= 0.9 ||
                   maxM_at(g, m, ix - 1, iy - 1, iz) <= 0.9;
  if (vac) return;
  // B is the predictor's con2prim when the divisors agree bit for bit
  // (k_update<true> stored it in pBC); otherwise computed here
  const bool haveB = (clk[0] + dt) - dt == clk[0];
#pragma unroll 1
  for (int w = haveB ? 1 : 0; w < 2; w++) {
    const double* src = w == 0 ? Qprev : Q;
    const double tt = w == 0 ? tau - dt : tau;
    double qs[7];
#pragma unroll
    for (int k = 0; k < 7; k++) qs[k] = src[k * N + i];
    q_over(qs, tt, q);
    Prim P;
    transform_pv<EK>(E, q, P, c2p_guess(E, i));
    const double ut = 1.0 / sqrt(1.0 - P.vx * P.vx - P.vy * P.vy - P.vz * P.vz);
    const int o = w == 0 ? 0 : 5;
    pBC[(o + 0) * N + i] = ut;
    pBC[(o + 1) * N + i] = ut * P.vx;
    pBC[(o + 2) * N + i] = ut * P.vy;
    pBC[(o + 3) * N + i] = ut * P.vz;
    if (w == 0) pBC[4 * N + i] = P.e;
  }
}
template <int EK>
__global__ void __launch_bounds__(128, 8) k_visc_prims(Geo g, EosDev E, TrDev tr,
                                                    const double* __restrict__ Q,
                                                    const double* __restrict__ Qprev,
                                                    const double* __restrict__ Qh,
                                                    const double* __restrict__ m,
                                                    double* __restrict__ pA,
                                                    double* __restrict__ pD,
                                                    double* __restrict__ pTh,
                                                    double* __restrict__ pBC, const double* __restrict__ clk,
                                                    const unsigned char* __restrict__ isdst) {
  d_visc_prims<EK>(g, E, tr, Q, Qprev, Qh, m, pA, pD, pTh, pBC, clk, isdst, blockIdx.x);
}


__device__ __forceinline__ double maxM_at(const Geo& g, const double* __restrict__ m, int ix,
                                          int iy, int iz) {
  return maxM(m, g.N, cidx(g, ix, iy, iz));
}

__device__ __forceinline__ Prim loadA(const double* __restrict__ pA, long long N, long long i) {
  Prim a;
  a.e = pA[i];
  a.p = pA[N + i];
  a.nb = pA[2 * N + i];
  a.nq = pA[3 * N + i];
  a.ns = pA[4 * N + i];
  a.vx = pA[5 * N + i];
  a.vy = pA[6 * N + i];
  a.vz = pA[7 * N + i];
  return a;
}

// ------------------------------------------------ ISformal, loop #1
// Hydro::ISformal loop 1 with Hydro::NSquant (src/hdo.cpp:381-652,
// 690-864): Navier-Stokes shear/bulk from the velocity gradients, then the
// two-stage Israel-Stewart relaxation with Christoffel and cross terms.
// Writes pi0/piH0/Pi0/PiH0 and the first flux contribution
// (+(tau-dt) * delta Q_n).  One thread per cell, every index a compile-time
// constant; the con2prims and the thermodynamics come precomputed from
// k_visc_prims.  Four 128-thread blocks per SM (128 registers) hide the FP64
// latency better than fewer, spill-free ones (measured: 3 and 2 blocks per SM
// are 7 % and 35 % slower, 5 and 6 are 9 % and 3 % slower).
constexpr int kRelaxMinBlocks = 4;

constexpr int kRelaxBlock = 128;
// shared-memory rows of k_is_relax's relaxation loops: pi, sigma, u, h0, f0,
// and phi7 h0^{kl} - tau_pipi sigma^{kl} of the second loop (dynamic shared
// memory: 55 KB per block, four blocks per SM)
constexpr int kSmPI = 0, kSmSIG = 10, kSmU = 20, kSmH = 24, kSmF = 34, kSmY = 44, kSmRows = 54;
constexpr size_t kRelaxSmem = sizeof(double) * kSmRows * kRelaxBlock;

// The empty cells' share of ISformal loop 1 (src/hdo.cpp:697-708: zero
// pi0/piH0/Pi0/PiH0) and the list of the other cells, so that k_is_relax
// runs full warps: cells with matter are packed in warp order (one atomic
// per warp; the list's order between warps varies, and every cell's result
// depends on that cell alone).  *nactive is zero on entry.
__device__ __forceinline__ void d_relax_list(const Geo& g, const double* __restrict__ pA,
                                             int* __restrict__ active, int* __restrict__ nactive,
                                             double* __restrict__ pi0, double* __restrict__ piH0,
                                             double* __restrict__ Pi0, double* __restrict__ PiH0,
                                             double* __restrict__ flux, long long blk) {
  const long long i = blk * blockDim.x + threadIdx.x;
  const long long N = g.N;
  const bool in = i < N;
  const bool act = in && !(pA[i] <= 0.);
  const int lane = threadIdx.x & 31;
  const unsigned bal = __ballot_sync(0xffffffffu, act);
  int base = 0;
  if (lane == 0 && bal) base = atomicAdd(nactive, __popc(bal));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (act) active[base + __popc(bal & ((1u << lane) - 1u))] = (int)i;
  if (in && !act) {
#pragma unroll
    for (int k = 0; k < 10; k++) {
      piH0[k * N + i] = 0.0;
      pi0[k * N + i] = 0.0;
    }
    PiH0[i] = 0.0;
    Pi0[i] = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) flux[k * N + i] = 0.;
  }
}
__global__ void __launch_bounds__(128) k_relax_list(Geo g, const double* __restrict__ pA,
                                                    int* __restrict__ active,
                                                    int* __restrict__ nactive,
                                                    double* __restrict__ pi0,
                                                    double* __restrict__ piH0,
                                                    double* __restrict__ Pi0,
                                                    double* __restrict__ PiH0,
                                                    double* __restrict__ flux) {
  d_relax_list(g, pA, active, nactive, pi0, piH0, Pi0, PiH0, flux, blockIdx.x);
}


__device__ __forceinline__ void d_is_relax(
    const Geo& g, const EosDev& E, const TrDev& tr, const double* __restrict__ Q,
    const double* __restrict__ Qprev, const double* __restrict__ m, const double* __restrict__ pA,
    const double* __restrict__ pD, const double* __restrict__ pTh,
    const double* __restrict__ pBC, const double* __restrict__ pi, const double* __restrict__ Pi,
    double* __restrict__ pi0, double* __restrict__ piH0, double* __restrict__ Pi0,
    double* __restrict__ PiH0, double* __restrict__ flux, const double* __restrict__ clk,
    unsigned* err, const int* __restrict__ active, const int* __restrict__ nactive,
    long long blk) {
  const double dt = clk[1], tau = clk[0] + dt;  // tau_{n+1} (src/hdo.cpp:1095)
  const int idx = (int)(blk * blockDim.x + threadIdx.x);
  if (idx >= *nactive) return;
  const long long i = active[idx];  // a cell with matter (k_relax_list)
  const long long N = g.N;
  const double e = pA[i];
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  const double gmumu[4] = {1., -1., -1., -1.};
  double cpi[10];
#pragma unroll
  for (int k = 0; k < 10; k++) cpi[k] = pi[k * N + i];
  const double cPi = Pi[i];
#define PI(a, b) cpi[index44(a, b)]
  const double vx = pA[5 * N + i], vy = pA[6 * N + i], vz = pA[7 * N + i];
  const double gamma = 1.0 / sqrt(1.0 - vx * vx - vy * vy - vz * vz);
  // the ~600 divisions by gamma go through crm::mk_div (bit-identical to
  // the divide) in batches whose numerators are all in its range
  const double rg = 1.0 / gamma;
  const bool gfast = crm::mk_den_ok(gamma);
  double u[4];
  u[0] = gamma;
  u[1] = u[0] * vx;
  u[2] = u[0] * vy;
  u[3] = u[0] * vz;
  {
    double f[4];
#pragma unroll
    for (int k = 0; k < 4; k++) f[k] = (tau - dt) * (PI(0, k) + cPi * u[0] * u[k]);
    f[0] += -(tau - dt) * cPi;
#pragma unroll
    for (int k = 0; k < 4; k++) flux[k * N + i] = 0. + f[k];
  }
  const double s = pTh[3 * N + i];
  const double etaS = pTh[4 * N + i];
  const double zetaS = pTh[5 * N + i];

  // ------------------------------------------------------ NSquant
  double piNS[10], PiNS, du;
  double dmu[4][4];
  const bool vac = maxM(m, N, cidx(g, ix + 1, iy, iz)) <= 0.9 ||
                   maxM(m, N, cidx(g, ix, iy + 1, iz)) <= 0.9 ||
                   maxM(m, N, cidx(g, ix - 1, iy, iz)) <= 0.9 ||
                   maxM(m, N, cidx(g, ix, iy - 1, iz)) <= 0.9 ||
                   maxM(m, N, cidx(g, ix + 1, iy + 1, iz)) <= 0.9 ||
                   maxM(m, N, cidx(g, ix + 1, iy - 1, iz)) <= 0.9 ||
                   maxM(m, N, cidx(g, ix - 1, iy + 1, iz)) <= 0.9 ||
                   maxM(m, N, cidx(g, ix - 1, iy - 1, iz)) <= 0.9;
  if (vac) {
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) dmu[a][b] = 0.;
#pragma unroll
    for (int k = 0; k < 10; k++) piNS[k] = 0.;
    PiNS = du = 0.;
  } else {
    const double VMIN = 1e-2;
    const double UDIFF = 3.0;
    const double e0 = pBC[4 * N + i], e1 = e;
    double ut0 = pBC[0 * N + i], ux0 = pBC[1 * N + i], uy0 = pBC[2 * N + i], uz0 = pBC[3 * N + i];
    double ut1 = pBC[5 * N + i], ux1 = pBC[6 * N + i], uy1 = pBC[7 * N + i], uz1 = pBC[8 * N + i];
    const double* uuu = u;
    dmu[0][0] = ddivp(ddivp((ut1 * ut1 - ut0 * ut0) / 2., uuu[0]), dt);
    dmu[0][1] = ddivp(ddiv((ux1 * ux1 - ux0 * ux0) / 2., uuu[1]), dt);
    dmu[0][2] = ddivp(ddiv((uy1 * uy1 - uy0 * uy0) / 2., uuu[2]), dt);
    dmu[0][3] = ddivp(ddiv((uz1 * uz1 - uz0 * uz0) / 2., uuu[3]), dt);
    if (fabs(ddivp(0.5 * (ut1 + ut0), ut1)) > UDIFF) dmu[0][0] = ddivp(ut1 - ut0, dt);
    if (fabs(uuu[1]) < VMIN || fabs(ddiv(0.5 * (ux1 + ux0), ux1)) > UDIFF)
      dmu[0][1] = ddivp(ux1 - ux0, dt);
    if (fabs(uuu[2]) < VMIN || fabs(ddiv(0.5 * (uy1 + uy0), uy1)) > UDIFF)
      dmu[0][2] = ddivp(uy1 - uy0, dt);
    if (fabs(uuu[3]) < VMIN || fabs(ddiv(0.5 * (uz1 + uz0), uz1)) > UDIFF)
      dmu[0][3] = ddivp(uz1 - uz0, dt);
    if (e1 <= 0. || e0 <= 0.) dmu[0][0] = dmu[0][1] = dmu[0][2] = dmu[0][3] = 0.;
#pragma unroll
    for (int d = 1; d <= 3; d++) {
      long long ip, im;
      if (d == 1) {
        ip = cidx(g, ix + 1, iy, iz);
        im = cidx(g, ix - 1, iy, iz);
      } else if (d == 2) {
        ip = cidx(g, ix, iy + 1, iz);
        im = cidx(g, ix, iy - 1, iz);
      } else {
        ip = cidx(g, ix, iy, iz + 1);
        im = cidx(g, ix, iy, iz - 1);
      }
      const double ep = pD[ip], em = pD[im];
      if (ep > 0. && em > 0.) {
        const double vx1 = pD[N + ip], vy1 = pD[2 * N + ip], vz1 = pD[3 * N + ip];
        const double vx0 = pD[N + im], vy0 = pD[2 * N + im], vz0 = pD[3 * N + im];
        ut0 = 1.0 / sqrt(1.0 - vx0 * vx0 - vy0 * vy0 - vz0 * vz0);
        ux0 = ut0 * vx0;
        uy0 = ut0 * vy0;
        uz0 = ut0 * vz0;
        ut1 = 1.0 / sqrt(1.0 - vx1 * vx1 - vy1 * vy1 - vz1 * vz1);
        ux1 = ut1 * vx1;
        uy1 = ut1 * vy1;
        uz1 = ut1 * vz1;
        if (d < 3) {
          const double h = d == 1 ? g.dx : g.dy;
          dmu[d][0] = ddivp(ddivp(0.25 * (ut1 * ut1 - ut0 * ut0), uuu[0]), h);
          dmu[d][1] = ddivp(ddiv(0.25 * (ux1 * ux1 - ux0 * ux0), uuu[1]), h);
          dmu[d][2] = ddivp(ddiv(0.25 * (uy1 * uy1 - uy0 * uy0), uuu[2]), h);
          dmu[d][3] = ddivp(ddiv(0.25 * (uz1 * uz1 - uz0 * uz0), uuu[3]), h);
          if (fabs(ddivp(0.5 * (ut1 + ut0), uuu[0])) > UDIFF) dmu[d][0] = ddivp(0.5 * (ut1 - ut0), h);
          if (fabs(uuu[1]) < VMIN || fabs(ddiv(0.5 * (ux1 + ux0), uuu[1])) > UDIFF)
            dmu[d][1] = ddivp(0.5 * (ux1 - ux0), h);
          if (fabs(uuu[2]) < VMIN || fabs(ddiv(0.5 * (uy1 + uy0), uuu[2])) > UDIFF)
            dmu[d][2] = ddivp(0.5 * (uy1 - uy0), h);
          if (fabs(uuu[3]) < VMIN || fabs(ddiv(0.5 * (uz1 + uz0), uuu[3])) > UDIFF)
            dmu[d][3] = ddivp(0.5 * (uz1 - uz0), h);
        } else {
          const double dz = g.dz, th = tau + 0.5 * dt;
          dmu[3][0] = ddivp(ddivp(ddivp(0.25 * (ut1 * ut1 - ut0 * ut0), uuu[0]), dz), th);
          dmu[3][1] = ddivp(ddivp(ddiv(0.25 * (ux1 * ux1 - ux0 * ux0), uuu[1]), dz), th);
          dmu[3][2] = ddivp(ddivp(ddiv(0.25 * (uy1 * uy1 - uy0 * uy0), uuu[2]), dz), th);
          dmu[3][3] = ddivp(ddivp(ddiv(0.25 * (uz1 * uz1 - uz0 * uz0), uuu[3]), dz), th);
          if (fabs(ddivp(0.5 * (ut1 + ut0), uuu[0])) > UDIFF)
            dmu[3][0] = ddivp(ddivp(0.5 * (ut1 - ut0), dz), th);
          if (fabs(uuu[1]) < VMIN || fabs(ddiv(0.5 * (ux1 + ux0), uuu[1])) > UDIFF)
            dmu[3][1] = ddivp(ddivp(0.5 * (ux1 - ux0), dz), th);
          if (fabs(uuu[2]) < VMIN || fabs(ddiv(0.5 * (uy1 + uy0), uuu[2])) > UDIFF)
            dmu[3][2] = ddivp(ddivp(0.5 * (uy1 - uy0), dz), th);
          if (fabs(uuu[3]) < VMIN || fabs(ddiv(0.5 * (uz1 + uz0), uuu[3])) > UDIFF)
            dmu[3][3] = ddivp(ddivp(0.5 * (uz1 - uz0), dz), th);
        }
      } else {
        dmu[d][0] = dmu[d][1] = dmu[d][2] = dmu[d][3] = 0.;
      }
    }
    dmu[3][0] += ddivp(uuu[3], tau - 0.5 * dt);
    dmu[3][3] += ddivp(uuu[0], tau - 0.5 * dt);
    const double gdiag[4] = {1., -1., -1., -1.};
    const double r5068 = 1.0 / 5.068;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b <= a; b++) {
        double n[16];  // the (k, l) terms, divided by 5.068 as a batch
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
          for (int l = 0; l < 4; l++) {
            double Z = 0.0;
            const double gak = (a == k) ? gdiag[a] : 0.;
            const double gbk = (b == k) ? gdiag[b] : 0.;
            const double gab = (a == b) ? gdiag[a] : 0.;
            if (b == l) Z += 0.5 * (gak - uuu[a] * uuu[k]);
            if (a == l) Z += 0.5 * (gbk - uuu[b] * uuu[k]);
            if (k == l) Z -= ddivp(gab - uuu[a] * uuu[b], 3.0);
            n[4 * k + l] = Z * dmu[k][l] * 2.0 * etaS * s;
          }
        div_batch<16>(n, 5.068, r5068, true);
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < 16; j++) acc += n[j];
        piNS[index44(a, b)] = acc;
      }
    PiNS = ddivp(-zetaS * s * (dmu[0][0] + dmu[1][1] + dmu[2][2] + dmu[3][3]), 5.068);
    du = dmu[0][0] + dmu[1][1] + dmu[2][2] + dmu[3][3];
    bool bad = false;
#pragma unroll
    for (int k = 0; k < 10; k++) bad |= isinf(piNS[k]) || isnan(piNS[k]);
    if (bad) atomicOr(err, (unsigned)ERR_NSQUANT_NAN);
  }
#define PINS(a, b) piNS[index44(a, b)]

  // ------------------------------------------------ ISformal loop 1 body
  const double eta = etaS * s;
  double sig[10];
#pragma unroll
  for (int k = 0; k < 10; k++) sig[k] = 0.5 * piNS[k];
  div_batch<10, true>(sig, eta, 1.0 / eta, crm::mk_den_ok(eta));  // ddiv's quotients
#pragma unroll
  for (int k = 0; k < 10; k++) {
    sig[k] = sig[k] * 5.068;
    if (eta <= 0.0) sig[k] = 0.0;
  }
#define SIG(a, b) sig[index44(a, b)]
  const double taupi = pTh[6 * N + i], tauPi = pTh[7 * N + i];
  double deltapipi = 4. / 3., taupipi = 10. / 7., lambdapiPi = 6. / 5.;
  double phi7 = pTh[8 * N + i];
  if (isinf(phi7)) phi7 = 0.0;
  phi7 = ddiv(phi7, taupi);
  if (taupi < 0.5 * dt) deltapipi = taupipi = lambdapiPi = phi7 = 0.0;
  double delPiPi = 2. / 3.;
  double lamPipi = 8. / 5. * (1. / 3. - 1. / 3.);
  if (tauPi < 0.5 * dt) delPiPi = lamPipi = 0.0;
  double Delta[10];
  double h0[10];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b <= a; b++) {
      const int k = index44(a, b);
      Delta[k] = -u[a] * u[b];
      if (a == b) Delta[k] += gmumu[a];
    }
  if (taupi > 0.5 * dt) {
    double n[10];
#pragma unroll
    for (int k = 0; k < 10; k++) n[k] = (cpi[k] - piNS[k]) * dt / 2.0;
    div_batch<10>(n, gamma, rg, gfast);
    div_batch<10>(n, taupi, 1.0 / taupi, crm::mk_den_ok(taupi));
#pragma unroll
    for (int k = 0; k < 10; k++) h0[k] = cpi[k] - n[k];
  } else {
#pragma unroll
    for (int k = 0; k < 10; k++) h0[k] = piNS[k];
  }
  double H0;
  if (tauPi > 0.5 * dt)
    H0 = cPi - ddivp(ddivp((cPi - PiNS) * dt / 2.0, gamma), tauPi);
  else
    H0 = PiNS;
  double tau1 = tau - dt * 0.75;
  h0[index44(0, 0)] += ddivp(-2. * vz * PI(0, 3), tau1) * dt / 2.;
  h0[index44(3, 3)] += -(ddivp(2. * vz, tau1) * PI(0, 3)) * dt / 2.;
  h0[index44(3, 0)] += -(ddivp(vz, tau1) * PI(0, 0) + ddivp(vz, tau1) * PI(3, 3)) * dt / 2.;
  h0[index44(1, 0)] += ddivp(-vz, tau1) * PI(1, 3) * dt / 2.;
  h0[index44(2, 0)] += ddivp(-vz, tau1) * PI(2, 3) * dt / 2.;
  h0[index44(3, 1)] += -(ddivp(vz, tau1) * PI(0, 1)) * dt / 2.;
  h0[index44(3, 2)] += -(ddivp(vz, tau1) * PI(0, 2)) * dt / 2.;
  // The relaxation sums over (a, b) run as a loop with (a, b) known only at
  // run time, so that its body (36 divisions by gamma) is fetched once per
  // warp instead of ten times unrolled: the unrolled kernel's instruction
  // stream outgrew the instruction caches.  Operands indexed by a or b come
  // from shared memory ([component][thread]); the arithmetic of every term
  // is the reference's, in its order.
  extern __shared__ double relax_smem[];
  double(*sm)[kRelaxBlock] = reinterpret_cast<double(*)[kRelaxBlock]>(relax_smem);
  const int t = threadIdx.x;
#pragma unroll
  for (int k = 0; k < 10; k++) {
    sm[kSmPI + k][t] = cpi[k];
    sm[kSmSIG + k][t] = sig[k];
    sm[kSmH + k][t] = h0[k];
  }
#pragma unroll
  for (int k = 0; k < 4; k++) sm[kSmU + k][t] = u[k];
  // phi7 pi^{kl} - tau_pipi sigma^{kl}, the same for every (a, b): in the
  // rows loop 2 uses for f0 later
#pragma unroll
  for (int k = 0; k < 10; k++) sm[kSmF + k][t] = phi7 * cpi[k] - taupipi * sig[k];
#pragma unroll 1
  for (int ab = 0; ab < 10; ab++) {
    const int a = ab >= 6 ? 3 : ab >= 3 ? 2 : ab >= 1 ? 1 : 0;
    const int b = ab - a * (a + 1) / 2;
    const double ua = sm[kSmU + a][t], ub = sm[kSmU + b][t];
    double dab = -ua * ub;  // Delta[index44(a, b)]
    if (a == b) dab += a == 0 ? 1. : -1.;
    double acc = sm[kSmH + ab][t];
    acc += ddivp(-deltapipi * sm[kSmPI + ab][t] * du + lambdapiPi * cPi * sm[kSmSIG + ab][t],
                 gamma) *
           0.5 * dt;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double gk = gmumu[k];
      const double pak = sm[kSmPI + index44(a, k)][t], pbk = sm[kSmPI + index44(b, k)][t];
      const double sak = sm[kSmSIG + index44(a, k)][t], sbk = sm[kSmSIG + index44(b, k)][t];
      double n[9];  // numerators of the k term and of its four (x, y) l terms
      n[0] = phi7 * pak * pbk * gk - taupipi * 0.5 * (pak * sbk * gk + pbk * sak * gk);
#pragma unroll
      for (int l = 0; l < 4; l++) {
        n[1 + 2 * l] = (-pak * ub - pbk * ua) * u[l] * dmu[l][k] * gk;
        n[2 + 2 * l] = 1. / 3. * dab * PI(k, l) * sm[kSmF + index44(k, l)][t] * gk * gmumu[l];
      }
      div_batch<9>(n, gamma, rg, gfast);
      acc += n[0] * 0.5 * dt;
#pragma unroll
      for (int l = 0; l < 4; l++) acc += n[1 + 2 * l] * 0.5 * dt - n[2 + 2 * l] * 0.5 * dt;
    }
    sm[kSmH + ab][t] = acc;
  }
#pragma unroll
  for (int k = 0; k < 10; k++) h0[k] = sm[kSmH + k][t];
  {
    double n[16];
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int l = 0; l < 4; l++) n[4 * k + l] = lamPipi * PI(k, l) * SIG(k, l) * gmumu[k] * gmumu[l];
    div_batch<16>(n, gamma, rg, gfast);
#pragma unroll
    for (int j = 0; j < 16; j++) H0 += n[j] * 0.5 * dt;
  }
  H0 += ddivp(-delPiPi * cPi * du, gamma) * 0.5 * dt;
#define H(a, b) h0[index44(a, b)]
  double f0[10];
  if (taupi > 0.5 * dt) {
    double n[10];
#pragma unroll
    for (int k = 0; k < 10; k++) n[k] = (h0[k] - piNS[k]) * dt;
    div_batch<10>(n, gamma, rg, gfast);
    div_batch<10>(n, taupi, 1.0 / taupi, crm::mk_den_ok(taupi));
#pragma unroll
    for (int k = 0; k < 10; k++) f0[k] = cpi[k] - n[k];
  } else {
#pragma unroll
    for (int k = 0; k < 10; k++) f0[k] = piNS[k];
  }
  double F0;
  if (tauPi > 0.5 * dt)
    F0 = cPi - ddivp(ddivp((H0 - PiNS) * dt, gamma), tauPi);
  else
    F0 = PiNS;
  tau1 = tau - dt * 0.5;
  f0[index44(0, 0)] += ddivp(-2. * vz, tau1) * H(0, 3) * dt;
  f0[index44(3, 3)] += -(ddivp(2. * vz, tau1) * H(0, 3)) * dt;
  f0[index44(3, 0)] += -(ddivp(vz, tau1) * H(0, 0) + ddivp(vz, tau1) * H(3, 3)) * dt;
  f0[index44(1, 0)] += ddivp(-vz, tau1) * H(1, 3) * dt;
  f0[index44(2, 0)] += ddivp(-vz, tau1) * H(2, 3) * dt;
  f0[index44(3, 1)] += -(ddivp(vz, tau1) * H(0, 1)) * dt;
  f0[index44(3, 2)] += -(ddivp(vz, tau1) * H(0, 2)) * dt;
#pragma unroll
  for (int k = 0; k < 10; k++) sm[kSmF + k][t] = f0[k];
#pragma unroll
  for (int k = 0; k < 10; k++) sm[kSmY + k][t] = phi7 * h0[k] - taupipi * sig[k];
#pragma unroll 1
  for (int ab = 0; ab < 10; ab++) {
    const int a = ab >= 6 ? 3 : ab >= 3 ? 2 : ab >= 1 ? 1 : 0;
    const int b = ab - a * (a + 1) / 2;
    const double ua = sm[kSmU + a][t], ub = sm[kSmU + b][t];
    double dab = -ua * ub;  // Delta[index44(a, b)]
    if (a == b) dab += a == 0 ? 1. : -1.;
    double acc = sm[kSmF + ab][t];
    acc += ddivp(-deltapipi * sm[kSmH + ab][t] * du + lambdapiPi * H0 * sm[kSmSIG + ab][t],
                 gamma) *
           dt;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double gk = gmumu[k];
      const double pak = sm[kSmPI + index44(a, k)][t];
      const double hak = sm[kSmH + index44(a, k)][t], hbk = sm[kSmH + index44(b, k)][t];
      const double sak = sm[kSmSIG + index44(a, k)][t], sbk = sm[kSmSIG + index44(b, k)][t];
      double n[5];  // numerators of the k term and of its four l terms
      n[0] = phi7 * pak * hbk * gk - taupipi * 0.5 * (hak * sbk * gk + hbk * sak * gk);
#pragma unroll
      for (int l = 0; l < 4; l++)
        n[1 + l] = (-hak * ub - hbk * ua) * u[l] * dmu[l][k] * gk -
                   1. / 3. * dab * H(k, l) * sm[kSmY + index44(k, l)][t] * gk * gmumu[l];
      div_batch<5>(n, gamma, rg, gfast);
      acc += n[0] * dt;
#pragma unroll
      for (int l = 0; l < 4; l++) acc += n[1 + l] * dt;
    }
    sm[kSmF + ab][t] = acc;
  }
#pragma unroll
  for (int k = 0; k < 10; k++) f0[k] = sm[kSmF + k][t];
  {
    double n[16];
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int l = 0; l < 4; l++) n[4 * k + l] = lamPipi * H(k, l) * SIG(k, l) * gmumu[k] * gmumu[l];
    div_batch<16>(n, gamma, rg, gfast);
#pragma unroll
    for (int j = 0; j < 16; j++) F0 += n[j] * dt;
  }
  F0 += ddivp(-delPiPi * H0 * du, gamma) * dt;
#pragma unroll
  for (int k = 0; k < 10; k++) {
    piH0[k * N + i] = h0[k];
    pi0[k * N + i] = f0[k];
  }
  PiH0[i] = H0;
  Pi0[i] = F0;
#undef PI
#undef PINS
#undef SIG
#undef H
}
__global__ void __launch_bounds__(kRelaxBlock, kRelaxMinBlocks) k_is_relax(
    Geo g, EosDev E, TrDev tr, const double* __restrict__ Q, const double* __restrict__ Qprev,
    const double* __restrict__ m, const double* __restrict__ pA, const double* __restrict__ pD,
    const double* __restrict__ pTh, const double* __restrict__ pBC,
    const double* __restrict__ pi, const double* __restrict__ Pi, double* __restrict__ pi0,
    double* __restrict__ piH0, double* __restrict__ Pi0, double* __restrict__ PiH0,
    double* __restrict__ flux, const double* __restrict__ clk, unsigned* err,
    const int* __restrict__ active, const int* __restrict__ nactive) {
  d_is_relax(g, E, tr, Q, Qprev, m, pA, pD, pTh, pBC, pi, Pi, pi0, piH0, Pi0, PiH0, flux, clk,
             err, active, nactive, blockIdx.x);
}


// ------------------------------------------------ ISformal, loop #2
// Semi-Lagrangian advection of pi0/piH0 from the 2x2x2 upwind cells, the
// viscous-correction limiter and the -(tau) * delta Q_{n+1} flux
// (src/hdo.cpp:866-962).
__device__ __forceinline__ double sgn(double x) {
  if (x > 0) return 1.;
  if (x < 0.) return -1.;
  return 0.;
}

__device__ __forceinline__ void d_is_advect(const Geo& g, const double* __restrict__ pA,
                                            const double* __restrict__ pi0,
                                            const double* __restrict__ piH0,
                                            const double* __restrict__ Pi0,
                                            const double* __restrict__ PiH0,
                                            double* __restrict__ pi, double* __restrict__ piH,
                                            double* __restrict__ Pi, double* __restrict__ PiH,
                                            double* __restrict__ vcc, double* __restrict__ flux,
                                            const double* __restrict__ clk,
                                            const int* __restrict__ active,
                                            const int* __restrict__ nactive, long long blk) {
  const double dt = clk[1], tau = clk[0] + dt;  // tau_{n+1} (src/hdo.cpp:1095)
  // the cells with matter only (k_relax_list); the empty ones are left as
  // they are, as the reference's loop 2 leaves them (e <= 0)
  const int idx = (int)(blk * blockDim.x + threadIdx.x);
  if (idx >= *nactive) return;
  const long long i = active[idx];
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  const long long N = g.N;
  const Prim A = loadA(pA, N, i);
  const double e = A.e, p = A.p, vx = A.vx, vy = A.vy, vz = A.vz;
  const double xm = ddivp(-vx * dt, g.dx);
  const double ym = ddivp(-vy * dt, g.dy);
  const double zm = ddivp(ddivp(-vz * dt, g.dz), tau - 0.5 * dt);
  const double xmH = ddivp(-vx * dt, g.dx) / 2.0;
  const double ymH = ddivp(-vy * dt, g.dy) / 2.0;
  const double zmH = ddivp(ddivp(-vz * dt, g.dz), tau - 0.5 * dt) / 2.0;
  const double wx[2] = {(1. - fabs(xm)), fabs(xm)};
  const double wy[2] = {(1. - fabs(ym)), fabs(ym)};
  const double wz[2] = {(1. - fabs(zm)), fabs(zm)};
  const double wxH[2] = {(1. - fabs(xmH)), fabs(xmH)};
  const double wyH[2] = {(1. - fabs(ymH)), fabs(ymH)};
  const double wzH[2] = {(1. - fabs(zmH)), fabs(zmH)};
  const int sx = (int)sgn(xm), sy = (int)sgn(ym), sz = (int)sgn(zm);
  double a[10], aH[10], P = 0.0, PH = 0.0;
#pragma unroll
  for (int k = 0; k < 10; k++) a[k] = aH[k] = 0.0;
#pragma unroll
  for (int jx = 0; jx < 2; jx++)
#pragma unroll
    for (int jy = 0; jy < 2; jy++)
#pragma unroll
      for (int jz = 0; jz < 2; jz++) {
        const long long c1 = cidx(g, ix + jx * sx, iy + jy * sy, iz + jz * sz);
        const double w = wx[jx] * wy[jy] * wz[jz];
        const double wH = wxH[jx] * wyH[jy] * wzH[jz];
#pragma unroll
        for (int k = 0; k < 10; k++) {
          a[k] += w * pi0[k * N + c1];
          aH[k] += wH * piH0[k * N + c1];
        }
        P += w * Pi0[c1];
        PH += wH * PiH0[c1];
      }
  const double maxT0 = smax(ddivp(e + p, 1. - vx * vx - vy * vy - vz * vz) - p,
                            ddivp((e + p) * (vx * vx + vy * vy + vz * vz), 1. - vx * vx - vy * vy - vz * vz) + p);
  double maxpi = 0.;
#pragma unroll
  for (int k = 0; k < 10; k++)
    if (fabs(a[k]) > maxpi) maxpi = fabs(a[k]);
  bool rescaled = false;
  if (ddiv(maxT0, maxpi) < 1.0) {
#pragma unroll
    for (int k = 0; k < 10; k++) {
      a[k] = ddiv(0.1 * a[k] * maxT0, maxpi);
      aH[k] = ddiv(0.1 * aH[k] * maxT0, maxpi);
    }
    rescaled = true;
  }
  if (fabs(P) > p) {
    if (P != 0.) P = 1 * P / fabs(P) * p;
    if (PH != 0.) PH = 1 * PH / fabs(PH) * p;
    rescaled = true;
  }
  vcc[i] = rescaled ? ddiv(maxT0, maxpi) : 1.;
#pragma unroll
  for (int k = 0; k < 10; k++) {
    pi[k * N + i] = a[k];
    piH[k * N + i] = aH[k];
  }
  Pi[i] = P;
  PiH[i] = PH;
  const double gamma = 1.0 / sqrt(1.0 - vx * vx - vy * vy - vz * vz);
  double u[4];
  u[0] = gamma;
  u[1] = u[0] * vx;
  u[2] = u[0] * vy;
  u[3] = u[0] * vz;
  double f[4];
#pragma unroll
  for (int k = 0; k < 4; k++) f[k] = -tau * (a[index44(0, k)] + P * u[0] * u[k]);
  f[0] += tau * P;
#pragma unroll
  for (int k = 0; k < 4; k++) flux[k * N + i] += f[k];
}
__global__ void __launch_bounds__(128) k_is_advect(Geo g, const double* __restrict__ pA,
                                                   const double* __restrict__ pi0,
                                                   const double* __restrict__ piH0,
                                                   const double* __restrict__ Pi0,
                                                   const double* __restrict__ PiH0,
                                                   double* __restrict__ pi, double* __restrict__ piH,
                                                   double* __restrict__ Pi, double* __restrict__ PiH,
                                                   double* __restrict__ vcc,
                                                   double* __restrict__ flux, const double* __restrict__ clk,
                                                   const int* __restrict__ active,
                                                   const int* __restrict__ nactive) {
  d_is_advect(g, pA, pi0, piH0, Pi0, PiH0, pi, piH, Pi, PiH, vcc, flux, clk, active, nactive,
              blockIdx.x);
}


// --------------------------------------------- viscous flux + update
// Hydro::visc_flux (src/hdo.cpp:966-1014) for the six faces of the cell,
// visc_source_step (src/hdo.cpp:355-375) and Cell::updateByViscFlux
// (src/cll.cpp:76-84).
// the face's cell size along dir (eta: dz (tau + dt/2), src/hdo.cpp:971-976)
__device__ __forceinline__ double visc_dxa(int dir, double tau, double dt, const Geo& g) {
  if (dir == X_) return g.dx;
  if (dir == Y_) return g.dy;
  return g.dz * (tau + 0.5 * dt);
}

// rdxa = RN(1 / dxa): the four quotients by dxa go through div_batch
__device__ __forceinline__ bool visc_face(int dir, double tau, double dt, const Geo& g,
                                          const double* __restrict__ pA,
                                          const double* __restrict__ piH,
                                          const double* __restrict__ PiH,
                                          const double* __restrict__ m, long long L, long long R,
                                          double dxa, double rdxa, double f[4]) {
  const long long N = g.N;
  if (m[(dir - 1) * N + L] < 1. && m[(dir - 1) * N + R] < 1.) return false;
  double vxl = pA[5 * N + L], vyl = pA[6 * N + L], vzl = pA[7 * N + L];
  const double vxr = pA[5 * N + R], vyr = pA[6 * N + R], vzr = pA[7 * N + R];
  vxl = 0.5 * (vxl + vxr);
  vyl = 0.5 * (vyl + vyr);
  vzl = 0.5 * (vzl + vzr);
  const double v = sqrt(vxl * vxl + vyl * vyl + vzl * vzl);
  if (v > 1.) {
    vxl = ddivp(0.99 * vxl, v);
    vyl = ddivp(0.99 * vyl, v);
    vzl = ddivp(0.99 * vzl, v);
  }
  const double gamma = 1. / sqrt(1. - v * v);
  const double uuu[4] = {gamma, gamma * vxl, gamma * vyl, gamma * vzl};
  const double gmumu[4] = {1., -1., -1., -1.};
  const double PL = PiH[L], PR = PiH[R];
#pragma unroll
  for (int a = 0; a < 4; a++) {
    const int k = index44(a, dir);
    double x = 0.5 * (piH[k * N + L] + piH[k * N + R]);
    if (a == dir) x += -0.5 * (PL + PR) * gmumu[a];
    x += 0.5 * (PL + PR) * uuu[a] * uuu[dir];
    f[a] = x * (tau - 0.5 * dt) * dt;
  }
  div_batch<4>(f, dxa, rdxa, crm::mk_den_ok(dxa));
  return true;
}

__device__ __forceinline__ void d_visc_update(const Geo& g, const double* __restrict__ pA,
                                              const double* __restrict__ piH,
                                              const double* __restrict__ PiH,
                                              const double* __restrict__ m,
                                              const double* __restrict__ flux,
                                              double* __restrict__ Q,
                                              const double* __restrict__ clk, long long blk) {
  const double dt = clk[1], tau = clk[0] + dt;  // tau_{n+1} (src/hdo.cpp:1095)
  const long long i = blk * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  const long long N = g.N;
  double fl[4];
#pragma unroll
  for (int k = 0; k < 4; k++) fl[k] = flux[k * N + i];
  double f[4];
  const long long st[3] = {1, g.nx, (long long)g.nx * g.ny};
  const int cc[3] = {ix, iy, iz};
  const int nn[3] = {g.nx, g.ny, g.nz};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double dxa = visc_dxa(d + 1, tau, dt, g), rdxa = 1.0 / dxa;
    if (cc[d] > 0 && visc_face(d + 1, tau, dt, g, pA, piH, PiH, m, i - st[d], i, dxa, rdxa, f)) {
#pragma unroll
      for (int k = 0; k < 4; k++) fl[k] += f[k];
    }
    if (cc[d] < nn[d] - 1 &&
        visc_face(d + 1, tau, dt, g, pA, piH, PiH, m, i, i + st[d], dxa, rdxa, f)) {
#pragma unroll
      for (int k = 0; k < 4; k++) fl[k] += -f[k];
    }
  }
  const double e = pA[i];
  if (!(e <= 0.)) {
    const double vx = pA[5 * N + i], vy = pA[6 * N + i], vz = pA[7 * N + i];
    double uuu[4];
    uuu[0] = 1. / sqrt(1. - vx * vx - vy * vy - vz * vz);
    uuu[1] = uuu[0] * vx;
    uuu[2] = uuu[0] * vy;
    uuu[3] = uuu[0] * vz;
    const double PH = PiH[i];
    double k0 = -piH[index44(3, 3) * N + i] + PH * (-1.0 - uuu[3] * uuu[3]);
    double k3 = -(piH[index44(0, 3) * N + i] + PH * uuu[0] * uuu[3]);
    k0 *= dt;
    k3 *= dt;
    fl[0] += k0;
    fl[1] += 0. * dt;
    fl[2] += 0. * dt;
    fl[3] += k3;
  }
  const double q0 = Q[i];
  if (fabs(fl[0]) <= 0.5 * q0) {
#pragma unroll
    for (int k = 0; k < 4; k++) Q[k * N + i] += fl[k];
#pragma unroll
    for (int k = 4; k < 7; k++) Q[k * N + i] += 0.;
  } else if (fl[0] != 0.) {
    const double fac = fabs(ddiv(0.5 * q0, fl[0]));
#pragma unroll
    for (int k = 0; k < 4; k++) Q[k * N + i] += fac * fl[k];
#pragma unroll
    for (int k = 4; k < 7; k++) Q[k * N + i] += fac * 0.;
  }
}
__global__ void __launch_bounds__(128, 8) k_visc_update(Geo g, const double* __restrict__ pA,
                                                     const double* __restrict__ piH,
                                                     const double* __restrict__ PiH,
                                                     const double* __restrict__ m,
                                                     const double* __restrict__ flux,
                                                     double* __restrict__ Q, const double* __restrict__ clk) {
  d_visc_update(g, pA, piH, PiH, m, flux, Q, clk, blockIdx.x);
}


// --------------------------------------------------- batched transformPV
__global__ void k_transform_pv(EosDev E, const double* __restrict__ Q, long long n,
                               double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double q[7];
#pragma unroll
  for (int k = 0; k < 7; k++) q[k] = Q[k * n + i];
  Prim o;
  transform_pv(E, q, o);
  out[0 * n + i] = o.e;
  out[1 * n + i] = o.p;
  out[2 * n + i] = o.nb;
  out[3 * n + i] = o.nq;
  out[4 * n + i] = o.ns;
  out[5 * n + i] = o.vx;
  out[6 * n + i] = o.vy;
  out[7 * n + i] = o.vz;
}

// ------------------------------------------------------------ launcher
static inline unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

const char* const kKernelNames[KK_COUNT] = {
    "k_update_m", "k_face_x", "k_face_y", "k_face_z", "k_update", "k_ghost",
    "k_visc_prims", "k_is_relax", "k_is_advect", "k_visc_update",
    "vorticity (k_vort_*, 6 kernels)"};


template <int EK>
static int launch_step_ek(const StepArgs& a, cudaStream_t s, LaunchMarker* mk) {
  const Geo& g = a.g;
  const int bs = a.block == 64 ? 64 : 128;
  const unsigned nb = nblk(g.N, bs);
  const unsigned nb128 = nblk(g.N, 128);
  int launches = 0;
  const Fields& F = a.f;
  auto done = [&](int kind) {
    launches++;
    if (mk) mk->after(kind);
  };
  k_update_m<<<nb, bs, 0, s>>>(g, F.m, F.m2, a.clk);
  done(KK_UPDATE_M);
  const double* m = F.m2;  // the updated fill fractions
  // predictor (src/hdo.cpp:1023-1060) and corrector (src/hdo.cpp:1062-1094)
  for (int pass = 0; pass < 2; pass++) {
    const bool pred = pass == 0;
    const double* QQ = pred ? F.Q : F.Qh;
    if (pred) {
      k_face<X_, true, EK><<<nb, bs, 0, s>>>(g, a.eos, QQ, m, F.Fx, a.clk, F.err);
      done(KK_FACE_X);
      k_face<Y_, true, EK><<<nb, bs, 0, s>>>(g, a.eos, QQ, m, F.Fy, a.clk, F.err);
      done(KK_FACE_Y);
      if (g.nz > 1) {
        k_face<Z_, true, EK><<<nb, bs, 0, s>>>(g, a.eos, QQ, m, F.Fz, a.clk, F.err);
        done(KK_FACE_Z);
      }
      k_update<true, EK><<<nb, bs, 0, s>>>(g, a.eos, F.Q, F.Qh, F.Qprev, F.Fx, F.Fy, F.Fz, a.clk, F.err,
                                       a.viscous ? F.pBC : nullptr, nullptr);
      done(KK_UPDATE);
    } else {
      k_face<X_, false, EK><<<nb, bs, 0, s>>>(g, a.eos, QQ, m, F.Fx, a.clk, F.err);
      done(KK_FACE_X);
      k_face<Y_, false, EK><<<nb, bs, 0, s>>>(g, a.eos, QQ, m, F.Fy, a.clk, F.err);
      done(KK_FACE_Y);
      if (g.nz > 1) {
        k_face<Z_, false, EK><<<nb, bs, 0, s>>>(g, a.eos, QQ, m, F.Fz, a.clk, F.err);
        done(KK_FACE_Z);
      }
      k_update<false, EK><<<nb, bs, 0, s>>>(g, a.eos, F.Q, F.Qh, F.Qprev, F.Fx, F.Fy, F.Fz, a.clk, F.err,
                                        nullptr, a.viscous ? F.pA : nullptr);
      done(KK_UPDATE);
    }
  }
  k_ghost<false><<<nb, bs, 0, s>>>(g, F.gsrc, F.gdst, F.Q, F.Qh, F.pi, F.Pi);
  done(KK_GHOST);
  if (a.viscous) {
    k_visc_prims<EK><<<nb, bs, 0, s>>>(g, a.eos, a.tr, F.Q, F.Qprev, F.Qh, m, F.pA, F.pD, F.pTh,
                                   F.pBC, a.clk, F.gdst);
    done(KK_VISC_PRIMS);
    if (a.vort) {
      launches += launch_vorticity(a, s) - 1;
      done(KK_VORT);
    }
    // the relaxation on full warps of cells with matter (the list kernel's
    // time is counted with the relaxation's)
    cudaMemsetAsync(F.nactive, 0, sizeof(int), s);
    k_relax_list<<<nb128, 128, 0, s>>>(g, F.pA, F.active, F.nactive, F.pi0, F.piH0, F.Pi0,
                                       F.PiH0, F.flux);
    launches++;
    k_is_relax<<<nb128, kRelaxBlock, kRelaxSmem, s>>>(g, a.eos, a.tr, F.Q, F.Qprev, m, F.pA, F.pD, F.pTh,
                                             F.pBC, F.pi, F.Pi, F.pi0, F.piH0, F.Pi0, F.PiH0,
                                             F.flux, a.clk, F.err, F.active, F.nactive);
    done(KK_IS_RELAX);
    k_is_advect<<<nb, bs, 0, s>>>(g, F.pA, F.pi0, F.piH0, F.Pi0, F.PiH0, F.pi, F.piH, F.Pi, F.PiH,
                                  F.vcc, F.flux, a.clk, F.active, F.nactive);
    done(KK_IS_ADVECT);
    k_visc_update<<<nb, bs, 0, s>>>(g, F.pA, F.piH, F.PiH, m, F.flux, F.Q, a.clk);
    done(KK_VISC_UPDATE);
  }
  k_ghost<true><<<nb, bs, 0, s>>>(g, F.gsrc, F.gdst, F.Q, F.Qh, F.pi, F.Pi);
  done(KK_GHOST);
  return launches;
}

int launch_step(const StepArgs& a, cudaStream_t s, LaunchMarker* mk) {
  const bool chiral = a.eos.kind == 2;
  if (a.eos.kind == 3) return launch_step_ek<EK_TABLE3>(a, s, mk);  // EoS3f (no slope method)
  if (a.eos.kind == 6) return launch_step_ek<EK_AZH>(a, s, mk);     // EoSAZH (no slope method)
  if (a.eos.kind == 7) return launch_step_ek<EK_CMFE>(a, s, mk);    // EoSCMFe (no slope method)
  if (a.eos.slope)
    return chiral ? launch_step_ek<EK_CHIRAL_SL>(a, s, mk) : launch_step_ek<EK_TABLE_SL>(a, s, mk);
  return chiral ? launch_step_ek<EK_CHIRAL>(a, s, mk) : launch_step_ek<EK_TABLE>(a, s, mk);
}

void launch_transform_pv(const EosDev& E, const double* Q, long long n, double* out,
                         cudaStream_t s) {
  k_transform_pv<<<nblk(n, 128), 128, 0, s>>>(E, Q, n, out);
}

// TransportCoeff::getEta + getTau (src/trancoeff.cpp:68-100) on arrays:
// in[6][n] = e, nb, T, muB, s, p -> out[4][n] = eta/s, zeta/s, tau_pi, tau_Pi
__global__ void k_transport(TrDev tr, const double* __restrict__ in, long long n,
                            double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double e = in[i], nb = in[n + i], T = in[2 * n + i], mub = in[3 * n + i],
               s = in[4 * n + i], p = in[5 * n + i];
  double taupi, tauPi;
  tr_getTau(tr, e, nb, T, mub, s, p, taupi, tauPi);
  out[i] = tr_etaS(tr, e, nb, T, mub, s, p);
  out[n + i] = tr_zetaS(tr, e, T, s, p);
  out[2 * n + i] = taupi;
  out[3 * n + i] = tauPi;
}

void launch_transport(const TrDev& tr, const double* in, long long n, double* out,
                      cudaStream_t s) {
  k_transport<<<nblk(n, 128), 128, 0, s>>>(tr, in, n, out);
}

// EoS::eos with muS, EoS::p and EoS::s (nq = ns = 0) on arrays:
// e[n], nb[n] -> out[6][n] = p, T, muB, muS, p(), s
__global__ void k_eos_eval(EosDev E, const double* __restrict__ e, const double* __restrict__ nb,
                           long long n, double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double T, mub, mus, p;
  eos_eval(E, e[i], nb[i], T, mub, mus, p);
  out[i] = p;
  out[n + i] = T;
  out[2 * n + i] = mub;
  out[3 * n + i] = mus;
  out[4 * n + i] = eos_p(E, e[i], nb[i]);
  out[5 * n + i] = eos_s(E, e[i], nb[i], 0., 0.);
}

void launch_eos_eval(const EosDev& E, const double* e, const double* nb, long long n, double* out,
                     cudaStream_t s) {
  k_eos_eval<<<nblk(n, 128), 128, 0, s>>>(E, e, nb, n, out);
}

// ------------------------------------------------------------ clock
// The step kernels read (tau, dt) from a two-double device clock, so that a
// captured step stays valid from one step to the next.
__global__ void k_clock_set(double* clk, double tau, double dt) {
  clk[0] = tau;
  clk[1] = dt;
}
// tau += dt (src/hdo.cpp:1095), the substep divide (dt / n) and restore
// (dt * n) of the driver loop (src/main.cpp:411,415), in the host's order
__global__ void k_clock_op(double* clk, int op, int n) {
  if (op == 0)
    clk[0] += clk[1];
  else if (op == 1)
    clk[1] = clk[1] / n;
  else
    clk[1] = clk[1] * n;
}

// ------------------------------------------------- stage-batched step
// The step kernels' bodies over a work table: block b of the launch is
// block items[b].blk of event items[b].ev, whose arguments come from
// evs[items[b].ev] (the small structures copied into registers, the
// field pointers loaded once).  Each event's cells see exactly the
// operations of its own launch_step; events are independent, so the order
// of blocks across events does not matter.
#define VH_ITEM                              \
  const BItem it = items[blockIdx.x];        \
  const StepDev& A = evs[it.ev];             \
  const Geo g = A.g;                         \
  const long long blk = it.blk;

__global__ void kb_update_m(const StepDev* __restrict__ evs, const BItem* __restrict__ items) {
  VH_ITEM
  d_update_m(g, A.f.m, A.f.m2, A.clk, blk);
}

template <int DIR, bool PRED, int EK>
__global__ void __launch_bounds__(128, 7) kb_face(const StepDev* __restrict__ evs,
                                               const BItem* __restrict__ items) {
  VH_ITEM
  const EosDev E = A.eos;
  double* F = DIR == X_ ? A.f.Fx : (DIR == Y_ ? A.f.Fy : A.f.Fz);
  d_face<DIR, PRED, EK>(g, E, PRED ? A.f.Q : A.f.Qh, A.f.m2, F, A.clk, A.f.err, blk);
}

template <bool PRED, int EK>
__global__ void __launch_bounds__(128, 12) kb_update(const StepDev* __restrict__ evs,
                                                 const BItem* __restrict__ items) {
  VH_ITEM
  const EosDev E = A.eos;
  double* pB = PRED && A.viscous ? A.f.pBC : nullptr;
  double* pA = !PRED && A.viscous ? A.f.pA : nullptr;
  d_update<PRED, EK>(g, E, A.f.Q, A.f.Qh, A.f.Qprev, A.f.Fx, A.f.Fy, A.f.Fz, A.clk, A.f.err, pB,
                     pA, blk);
}

template <bool FULL>
__global__ void kb_ghost(const StepDev* __restrict__ evs, const BItem* __restrict__ items) {
  VH_ITEM
  d_ghost<FULL>(g, A.f.gsrc, A.f.gdst, A.f.Q, A.f.Qh, A.f.pi, A.f.Pi, blk);
}

template <int EK>
__global__ void __launch_bounds__(128, 8) kb_visc_prims(const StepDev* __restrict__ evs,
                                                     const BItem* __restrict__ items) {
  VH_ITEM
  const EosDev E = A.eos;
  const TrDev tr = A.tr;
  d_visc_prims<EK>(g, E, tr, A.f.Q, A.f.Qprev, A.f.Qh, A.f.m2, A.f.pA, A.f.pD, A.f.pTh,
                   A.f.pBC, A.clk, A.f.gdst, blk);
}

__global__ void kb_nactive_zero(const StepDev* __restrict__ evs, int nev) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < nev) *evs[e].f.nactive = 0;
}

__global__ void __launch_bounds__(128) kb_relax_list(const StepDev* __restrict__ evs,
                                                     const BItem* __restrict__ items) {
  VH_ITEM
  d_relax_list(g, A.f.pA, A.f.active, A.f.nactive, A.f.pi0, A.f.piH0, A.f.Pi0, A.f.PiH0,
               A.f.flux, blk);
}

__global__ void __launch_bounds__(kRelaxBlock, kRelaxMinBlocks) kb_is_relax(
    const StepDev* __restrict__ evs, const BItem* __restrict__ items) {
  VH_ITEM
  const EosDev E = A.eos;
  const TrDev tr = A.tr;
  d_is_relax(g, E, tr, A.f.Q, A.f.Qprev, A.f.m2, A.f.pA, A.f.pD, A.f.pTh, A.f.pBC, A.f.pi,
             A.f.Pi, A.f.pi0, A.f.piH0, A.f.Pi0, A.f.PiH0, A.f.flux, A.clk, A.f.err, A.f.active,
             A.f.nactive, blk);
}

__global__ void __launch_bounds__(128) kb_is_advect(const StepDev* __restrict__ evs,
                                                    const BItem* __restrict__ items) {
  VH_ITEM
  d_is_advect(g, A.f.pA, A.f.pi0, A.f.piH0, A.f.Pi0, A.f.PiH0, A.f.pi, A.f.piH, A.f.Pi,
              A.f.PiH, A.f.vcc, A.f.flux, A.clk, A.f.active, A.f.nactive, blk);
}

__global__ void __launch_bounds__(128, 8) kb_visc_update(const StepDev* __restrict__ evs,
                                                      const BItem* __restrict__ items) {
  VH_ITEM
  d_visc_update(g, A.f.pA, A.f.piH, A.f.PiH, A.f.m2, A.f.flux, A.f.Q, A.clk, blk);
}
#undef VH_ITEM

__global__ void kb_clock_op(const StepDev* __restrict__ evs, int nev, int op,
                            const int* __restrict__ ns) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nev) return;
  double* clk = evs[e].clk;
  const int n = ns ? ns[e] : 1;
  if (op == 0)
    clk[0] += clk[1];
  else if (op == 1)
    clk[1] = clk[1] / n;
  else
    clk[1] = clk[1] * n;
}

// launch_step_ek's stages in its order, over the work table
template <int EK>
static int launch_step_batched_ek(bool viscous, const StepDev* evs, int nev, const BItem* items,
                                  int nitems, cudaStream_t s) {
  const unsigned nb = (unsigned)nitems, ne = nblk(nev, 128);
  int launches = 0;
  kb_update_m<<<nb, kBatchBlock, 0, s>>>(evs, items);
  launches++;
  // predictor and corrector; z faces of 2+1D events return at once
  kb_face<X_, true, EK><<<nb, kBatchBlock, 0, s>>>(evs, items);
  kb_face<Y_, true, EK><<<nb, kBatchBlock, 0, s>>>(evs, items);
  kb_face<Z_, true, EK><<<nb, kBatchBlock, 0, s>>>(evs, items);
  kb_update<true, EK><<<nb, kBatchBlock, 0, s>>>(evs, items);
  kb_face<X_, false, EK><<<nb, kBatchBlock, 0, s>>>(evs, items);
  kb_face<Y_, false, EK><<<nb, kBatchBlock, 0, s>>>(evs, items);
  kb_face<Z_, false, EK><<<nb, kBatchBlock, 0, s>>>(evs, items);
  kb_update<false, EK><<<nb, kBatchBlock, 0, s>>>(evs, items);
  kb_ghost<false><<<nb, kBatchBlock, 0, s>>>(evs, items);
  launches += 9;
  if (viscous) {
    kb_visc_prims<EK><<<nb, kBatchBlock, 0, s>>>(evs, items);
    kb_nactive_zero<<<ne, 128, 0, s>>>(evs, nev);
    kb_relax_list<<<nb, kBatchBlock, 0, s>>>(evs, items);
    kb_is_relax<<<nb, kRelaxBlock, kRelaxSmem, s>>>(evs, items);
    kb_is_advect<<<nb, kBatchBlock, 0, s>>>(evs, items);
    kb_visc_update<<<nb, kBatchBlock, 0, s>>>(evs, items);
    launches += 6;
  }
  kb_ghost<true><<<nb, kBatchBlock, 0, s>>>(evs, items);
  return launches + 1;
}

int step_ek(const EosDev& E) {
  if (E.kind == 3) return EK_TABLE3;
  if (E.kind == 6) return EK_AZH;
  if (E.kind == 7) return EK_CMFE;
  const bool chiral = E.kind == 2;
  if (E.slope) return chiral ? EK_CHIRAL_SL : EK_TABLE_SL;
  return chiral ? EK_CHIRAL : EK_TABLE;
}

int launch_step_batched(int ek, bool viscous, const StepDev* evs, int nev, const BItem* items,
                        int nitems, cudaStream_t s) {
  switch (ek) {
    case EK_TABLE3: return launch_step_batched_ek<EK_TABLE3>(viscous, evs, nev, items, nitems, s);
    case EK_AZH: return launch_step_batched_ek<EK_AZH>(viscous, evs, nev, items, nitems, s);
    case EK_CMFE: return launch_step_batched_ek<EK_CMFE>(viscous, evs, nev, items, nitems, s);
    case EK_CHIRAL_SL:
      return launch_step_batched_ek<EK_CHIRAL_SL>(viscous, evs, nev, items, nitems, s);
    case EK_TABLE_SL:
      return launch_step_batched_ek<EK_TABLE_SL>(viscous, evs, nev, items, nitems, s);
    case EK_CHIRAL: return launch_step_batched_ek<EK_CHIRAL>(viscous, evs, nev, items, nitems, s);
    default: return launch_step_batched_ek<EK_TABLE>(viscous, evs, nev, items, nitems, s);
  }
}

void launch_clock_op_batched(const StepDev* evs, int nev, int op, const int* ns, cudaStream_t s) {
  kb_clock_op<<<nblk(nev, 128), 128, 0, s>>>(evs, nev, op, ns);
}

cudaError_t step_kernels_setup() {
  cudaError_t e = cudaFuncSetAttribute(k_is_relax, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kRelaxSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kb_is_relax, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)kRelaxSmem);
}

void launch_clock_set(double* clk, double tau, double dt, cudaStream_t s) {
  k_clock_set<<<1, 1, 0, s>>>(clk, tau, dt);
}
void launch_clock_op(double* clk, int op, int n, cudaStream_t s) {
  k_clock_op<<<1, 1, 0, s>>>(clk, op, n);
}

// ------------------------------------------------------- small helpers
__global__ void k_fill(double* __restrict__ p, long long n, double v) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// Cell::setQ (src/cll.h:75-80): a row with Q_t < 0 becomes zero.
__global__ void k_zero_negative_rows(double* __restrict__ Q, long long N) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  if (Q[i] < 0.) {
#pragma unroll
    for (int k = 0; k < 7; k++) Q[k * N + i] = 0.;
  }
}

void launch_fill(double* p, long long n, double v, cudaStream_t s) {
  if (n > 0) k_fill<<<nblk(n, 256), 256, 0, s>>>(p, n, v);
}

void launch_zero_negative_rows(double* Q, long long N, cudaStream_t s) {
  if (N > 0) k_zero_negative_rows<<<nblk(N, 256), 256, 0, s>>>(Q, N);
}

// expandGrid2x decimation (src/main.cpp:259-266): new cell (ix, iy, iz) takes
// the old cell 2*(i - n/2) + n/2 in x and y, clamped like Fluid::getCell, and
// the same iz.  ncomp component planes of N cells each.
__global__ void k_resize_gather(Geo g, const double* __restrict__ src, double* __restrict__ dst,
                                int ncomp) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  int sx = 2 * (ix - g.nx / 2) + g.nx / 2, sy = 2 * (iy - g.ny / 2) + g.ny / 2;
  sx = sx > 0 ? sx : 0;
  sx = sx < g.nx ? sx : g.nx - 1;
  sy = sy > 0 ? sy : 0;
  sy = sy < g.ny ? sy : g.ny - 1;
  const long long j = cidx(g, sx, sy, iz);
  for (int k = 0; k < ncomp; k++) dst[k * g.N + i] = src[k * g.N + j];
}

void launch_resize_gather(const Geo& g, const double* src, double* dst, int ncomp,
                          cudaStream_t s) {
  if (g.N > 0) k_resize_gather<<<nblk(g.N, 256), 256, 0, s>>>(g, src, dst, ncomp);
}

// Planes z0 .. z0 + nz - 1 of every listed field to or from one contiguous
// buffer laid out [field][component][plane][nx*ny] (pack = 1: fields ->
// buffer).  A z-plane of a component is contiguous (x fastest, then y),
// so a thread moves one double and consecutive threads move consecutive
// doubles of one plane.
__global__ void k_planes(PlaneFields pf, long long N, long long nxy, int z0, int nz,
                         double* __restrict__ buf, int pack) {
  const long long per = (long long)nz * nxy;  // doubles per component
  const long long total = per * pf.ncomp_total;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    long long c = t / per;
    const long long r = t - c * per;
    int f = 0;
    while (c >= pf.ncomp[f]) c -= pf.ncomp[f++];
    double* p = pf.p[f] + c * N + (long long)z0 * nxy + r;
    if (pack)
      buf[t] = *p;
    else
      *p = buf[t];
  }
}

void launch_planes(const PlaneFields& pf, long long N, long long nxy, int z0, int nz,
                   double* buf, bool pack, cudaStream_t s) {
  const long long total = (long long)nz * nxy * pf.ncomp_total;
  if (total <= 0) return;
  const long long blocks = std::min<long long>((total + 255) / 256, 148LL * 16);
  k_planes<<<(unsigned)blocks, 256, 0, s>>>(pf, N, nxy, z0, nz, buf, pack ? 1 : 0);
}

}  // namespace vh
