// vh_surface.cu -- what Fluid::outputSurface (src/fld.cpp:517-874) computes
// from the grid after a step: the interior totals (energy, baryon number,
// entropy, momentum, flow anisotropy sums).
//
// The totals are a deterministic two-level reduction: every thread forms its
// cell's 16 contributions exactly as the reference does (src/fld.cpp:544-604),
// each block reduces them in a fixed tree (warp shuffles, then one warp over
// the block's warps), and a single block adds the block partials in index
// order.  Results do not depend on scheduling, so repeated runs are
// bit-identical; against the reference's sequential sum they differ only by
// summation order and by the last bits of log/cosh/sinh/tanh.
#include <cuda_runtime.h>

#include "vh_physics.cuh"
#include "vh_step.cuh"
#include "vh_surface.cuh"

namespace vh {

// Fluid::getCMFvariables, src/fld.cpp:50-60
__device__ __forceinline__ void cmf_variables(const EosDev& E, const double* __restrict__ Q,
                                              long long N, long long i, double eta, double tau,
                                              Prim& P, double& Y) {
  double q[7];
#pragma unroll
  for (int k = 0; k < 7; k++) q[k] = ddivp(Q[k * N + i], tau);
  transform_pv(E, q, P);
  Y = eta + 1. / 2. * log((1. + P.vz) / (1. - P.vz));
  P.vx = P.vx * cosh(Y - eta) / cosh(Y);
  P.vy = P.vy * cosh(Y - eta) / cosh(Y);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

constexpr int kTotBlock = 256;

__global__ void __launch_bounds__(kTotBlock) k_totals(Geo g, EosDev E, const double* __restrict__ Q,
                                                      const double* __restrict__ pi,
                                                      const double* __restrict__ vcc, double tau,
                                                      double ecrit, double etamin, bool visc,
                                                      double* __restrict__ partial) {
  __shared__ double red[kTotBlock / 32][kTotals];
  const int nix = g.nx - 4, niy = g.ny - 4, niz = g.nz - 4;
  const long long nint = (nix > 0 && niy > 0 && niz > 0) ? (long long)nix * niy * niz : 0;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double c[kTotals];
#pragma unroll
  for (int k = 0; k < kTotals; k++) c[k] = 0.;
  if (t < nint) {
    // interior cell, z fastest like the reference loop (ix, iy outer)
    const int iz = 2 + (int)(t % niz);
    const int iy = 2 + (int)((t / niz) % niy);
    const int ix = 2 + (int)(t / ((long long)niz * niy));
    const long long N = g.N;
    const long long i = ix + (long long)g.nx * iy + (long long)g.nx * g.ny * iz;
    const double dz = g.dz;
    const double eta = etamin + iz * dz;
    Prim P;
    double vz;
    cmf_variables(E, Q, N, i, eta, tau, P, vz);
    const double e = P.e, vx = P.vx, vy = P.vy;
    double T, mub, p;
    eos_eval(E, e, P.nb, T, mub, p);
    double s = eos_s(E, e, P.nb, P.nq, P.ns);
    const double cosh_int = (sinh(eta + 0.5 * dz) - sinh(eta - 0.5 * dz)) / dz;
    const double sinh_int = (cosh(eta + 0.5 * dz) - cosh(eta - 0.5 * dz)) / dz;
    const double th = tanh(vz);
    const double den = 1. - vx * vx - vy * vy - th * th;
    c[0] = tau * (e + p) / den * (cosh_int - th * sinh_int) - tau * p * cosh_int;
    c[2] = Q[NB_ * N + i];
    c[3] = tau * P.nb * (cosh_int - th * sinh_int) / sqrt(den);
    c[1] = tau * (e + p) / den * (cosh(eta) - th * sinh(eta)) - tau * p * cosh(eta);
    const double pi00 = pi[index44(0, 0) * N + i], pi03 = pi[index44(0, 3) * N + i];
    const double pi01 = pi[index44(0, 1) * N + i];
    if (visc) c[1] = c[1] + (tau * pi00 * cosh(eta) + tau * pi03 * sinh(eta));
    if (e > ecrit) {
      c[14] = 1.;
      if (vcc[i] < 0.9) c[15] = 1.;
    }
    double deltas = 0.;
    if (visc) {
      const double gm[4] = {1., -1., -1., -1.};
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const double pab = pi[index44(a, b) * N + i];
          deltas += pab * pab * gm[a] * gm[b];
        }
    }
    if (T > 0.02) {
      s += 1.5 * deltas / ((e + p) * T);
      c[4] = tau * s * (cosh_int - th * sinh_int) / sqrt(den);
    }
    c[5] = tau * (e + p) * vx / den;
    if (iz > g.nz / 2 - 3 && iz < g.nz / 2 + 3) {
      c[8] = e * (fabs(vx) - fabs(vy));
      c[9] = e;
      c[7] = e / sqrt(1. - vx * vx - vy * vy);
      c[6] = e / sqrt(1. - vx * vx - vy * vy) * sqrt(vx * vx + vy * vy);
      c[12] = (e + p) / den * (vx * vx - vy * vy);
      c[13] = (e + p) / den * (vx * vx + vy * vy) + 2. * p;
    }
    c[10] = e / den * fabs(pi01);
    c[11] = e / den;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kTotals; k++) {
    const double v = warp_sum(c[k]);
    if (lane == 0) red[w][k] = v;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < kTotals; k++) {
      double v = lane < kTotBlock / 32 ? red[lane][k] : 0.;
      v = warp_sum(v);
      if (lane == 0) partial[(long long)blockIdx.x * kTotals + k] = v;
    }
  }
}

// Adds the block partials in index order (one block, fixed tree).
__global__ void __launch_bounds__(kTotBlock) k_totals_final(const double* __restrict__ partial,
                                                            int nblocks, double* __restrict__ out) {
  __shared__ double red[kTotBlock / 32][kTotals];
  double c[kTotals];
#pragma unroll
  for (int k = 0; k < kTotals; k++) c[k] = 0.;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < kTotals; k++) c[k] += partial[(long long)b * kTotals + k];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kTotals; k++) {
    const double v = warp_sum(c[k]);
    if (lane == 0) red[w][k] = v;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < kTotals; k++) {
      double v = lane < kTotBlock / 32 ? red[lane][k] : 0.;
      v = warp_sum(v);
      if (lane == 0) out[k] = v;
    }
  }
}

int totals_blocks(const Geo& g) {
  const int nix = g.nx - 4, niy = g.ny - 4, niz = g.nz - 4;
  const long long nint = (nix > 0 && niy > 0 && niz > 0) ? (long long)nix * niy * niz : 0;
  const long long nb = (nint + kTotBlock - 1) / kTotBlock;
  return nb > 0 ? (int)nb : 1;
}

void launch_totals(const Geo& g, const EosDev& E, const Fields& f, double tau, double ecrit,
                   double etamin, bool viscous, double* partial, double* out, cudaStream_t s) {
  const int nb = totals_blocks(g);
  k_totals<<<nb, kTotBlock, 0, s>>>(g, E, f.Q, f.pi, f.vcc, tau, ecrit, etamin, viscous, partial);
  k_totals_final<<<1, kTotBlock, 0, s>>>(partial, nb, out);
}

}  // namespace vh
