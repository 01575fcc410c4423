// vh_surface.cu -- what Fluid::outputSurface (src/fld.cpp:517-874) computes
// from the grid after a step: the interior totals (energy, baryon number,
// entropy, momentum, flow anisotropy sums) and the freeze-out hypersurface
// elements (Cornelius 4D, vh_cornelius.cuh) with their interpolated state.
//
// The totals are a deterministic two-level reduction: every thread forms its
// cell's 16 contributions exactly as the reference does (src/fld.cpp:544-604),
// each block reduces them in a fixed tree (warp shuffles, then one warp over
// the block's warps), and a single block adds the block partials in index
// order.  Results do not depend on scheduling, so repeated runs are
// bit-identical; against the reference's sequential sum they differ only by
// summation order and by the last bits of log/cosh/sinh/tanh.
#include <cuda_runtime.h>

#include "vh_cornelius.cuh"
#include "vh_physics.cuh"
#include "vh_step.cuh"
#include "vh_surface.cuh"

namespace vh {

// Fluid::getCMFvariables, src/fld.cpp:50-60
__device__ __forceinline__ void cmf_variables(const EosDev& E, const double* __restrict__ Q,
                                              long long N, long long i, double eta, double tau,
                                              Prim& P, double& Y) {
  double q[7], qs[7];
#pragma unroll
  for (int k = 0; k < 7; k++) qs[k] = Q[k * N + i];
  q_over(qs, tau, q);
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
  const int nix = g.nx - 4, niy = g.ny - 4, niz = g.zt1 - g.zt0;
  const long long nint = (nix > 0 && niy > 0 && niz > 0) ? (long long)nix * niy * niz : 0;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double c[kTotals];
#pragma unroll
  for (int k = 0; k < kTotals; k++) c[k] = 0.;
  if (t < nint) {
    // interior cell, z fastest like the reference loop (ix, iy outer)
    const int iz = g.zt0 + (int)(t % niz);
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
    const int izg = iz + g.zoff;  // the plane in the whole grid (Fluid's nz)
    if (izg > g.nzg / 2 - 3 && izg < g.nzg / 2 + 3) {
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
  const int nix = g.nx - 4, niy = g.ny - 4, niz = g.zt1 - g.zt0;
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

// ===================================================================
// Freeze-out hypersurface: the element part of Fluid::outputSurface
// (src/fld.cpp:606-842).  Stages, all on the context's stream:
//   1. k_surf_energy     e at tau (Q) and at tau - dt (Qprev) per cell
//   2. k_surf_count      straddling interior cubes per block
//   3. k_scan_excl       block offsets (one block)
//   4. k_surf_compact    straddling cube list in the reference's loop order
//   5. k_surf_cornelius  Cornelius, a warp per cube -> centroids, normals, counts
//   6. k_scan_excl       element offsets
//   7. k_surf_elements   one record per element (+ its sums' contributions)
//   8. k_sum_cols        deterministic sums of the contributions
// ===================================================================
namespace vh {

template <int EK>
__global__ void k_surf_energy(Geo g, EosDev E, const double* __restrict__ Q,
                              const double* __restrict__ Qprev, double tau, double taup,
                              double* __restrict__ eN, double* __restrict__ eP) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  // only corners of interior cubes: [2, n-2] on every axis
  if (ix < 2 || iy < 2 || iz < g.zc0 || ix > g.nx - 2 || iy > g.ny - 2 || iz > g.zc1) return;
  const long long N = g.N;
  double q[7], qs[7];
  Prim P;
  // Cell::getPrimVar / getPrimVarPrev, src/cll.cpp:90-95,214-220
#pragma unroll
  for (int k = 0; k < 7; k++) qs[k] = Q[k * N + i];
  q_over(qs, tau, q);
  transform_pv<EK>(E, q, P);
  eN[i] = P.e;
#pragma unroll
  for (int k = 0; k < 7; k++) qs[k] = Qprev[k * N + i];
  q_over(qs, taup, q);
  transform_pv<EK>(E, q, P);
  eP[i] = P.e;
}

__device__ __forceinline__ void load_cube(const Geo& g, const double* __restrict__ eN,
                                          const double* __restrict__ eP, int ix, int iy, int iz,
                                          double* hc) {
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const long long i = cidx(g, ix + (c >> 2), iy + ((c >> 1) & 1), iz + (c & 1));
    hc[8 + c] = eN[i];
    hc[c] = eP[i];
  }
}

__device__ __forceinline__ bool straddles(const double* hc, double e0) {
  int above = 0;
#pragma unroll
  for (int k = 0; k < 16; k++) above += hc[k] >= e0;
  return above != 0 && above != 16;
}

constexpr int kSurfBlock = 256;

__global__ void __launch_bounds__(kSurfBlock) k_surf_count(Geo g, const double* __restrict__ eN,
                                                           const double* __restrict__ eP,
                                                           double e0, long long ncube,
                                                           int* __restrict__ blk) {
  const long long t = (long long)blockIdx.x * kSurfBlock + threadIdx.x;
  int flag = 0;
  if (t < ncube) {
    int ix, iy, iz;
    double hc[16];
    cube_cell(g, t, ix, iy, iz);
    load_cube(g, eN, eP, ix, iy, iz, hc);
    flag = straddles(hc, e0);
  }
  const int c = __syncthreads_count(flag);
  if (threadIdx.x == 0) blk[blockIdx.x] = c;
}

// Exclusive prefix sum of a[0..n) in place by one block; *total = the sum.
constexpr int kScanBlock = 1024;
// With n_dev set, n = min(*n_dev, cap) is read on the device.
__global__ void __launch_bounds__(kScanBlock) k_scan_excl(int* __restrict__ a, int n,
                                                          int* __restrict__ total,
                                                          const int* __restrict__ n_dev,
                                                          int cap) {
  __shared__ long long part[kScanBlock];
  if (n_dev) n = min(*n_dev, cap);
  const int per = (n + kScanBlock - 1) / kScanBlock;
  const int b = threadIdx.x * per, e = min(n, b + per);
  long long s = 0;
  for (int i = b; i < e; i++) s += a[i];
  part[threadIdx.x] = s;
  __syncthreads();
  // Hillis-Steele inclusive scan of the chunk sums
  for (int o = 1; o < kScanBlock; o <<= 1) {
    const long long v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  long long run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (int i = b; i < e; i++) {
    const int v = a[i];
    a[i] = (int)run;
    run += v;
  }
  if (threadIdx.x == kScanBlock - 1) *total = (int)part[kScanBlock - 1];
}

__global__ void __launch_bounds__(kSurfBlock) k_surf_compact(Geo g, const double* __restrict__ eN,
                                                             const double* __restrict__ eP,
                                                             double e0, long long ncube,
                                                             const int* __restrict__ blkoff,
                                                             int* __restrict__ cubes, int cap) {
  __shared__ int woff[kSurfBlock / 32];
  const long long t = (long long)blockIdx.x * kSurfBlock + threadIdx.x;
  bool flag = false;
  if (t < ncube) {
    int ix, iy, iz;
    double hc[16];
    cube_cell(g, t, ix, iy, iz);
    load_cube(g, eN, eP, ix, iy, iz, hc);
    flag = straddles(hc, e0);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned bal = __ballot_sync(0xffffffffu, flag);
  if (lane == 0) woff[w] = __popc(bal);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int k = 0; k < kSurfBlock / 32; k++) {
      const int v = woff[k];
      woff[k] = s;
      s += v;
    }
  }
  __syncthreads();
  const int slot = blkoff[blockIdx.x] + woff[w] + __popc(bal & ((1u << lane) - 1u));
  if (flag && slot < cap) cubes[slot] = (int)t;  // past cap: the host grows and reruns
}

constexpr int kGeo = 8;  // centroid[4], normal[4] per element

// One warp per straddling hypercube (vh_cornelius.cuh), two per block.
constexpr int kCornWarps = 2;

__global__ void __launch_bounds__(32 * kCornWarps) k_surf_cornelius(
    Geo g, const double* __restrict__ eN, const double* __restrict__ eP, double e0, double dt4,
    const int* __restrict__ cubes, const int* __restrict__ ncubes_dev, int cap,
    double* __restrict__ geo, int* __restrict__ cnt, unsigned* err) {
  __shared__ cnw::WarpWork ws[kCornWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ncubes = min(*ncubes_dev, cap);
  cnw::WarpWork& w = ws[warp];
  for (int k = blockIdx.x * kCornWarps + warp; k < ncubes; k += gridDim.x * kCornWarps) {
    int ix, iy, iz;
    cube_cell(g, cubes[k], ix, iy, iz);
    if (lane < 16) {  // corner it*8 + c: Qprev layer (it = 0) or Q layer (it = 1)
      const int c = lane & 7;
      const long long i = cidx(g, ix + (c >> 2), iy + ((c >> 1) & 1), iz + (c & 1));
      w.hc[lane] = (lane >> 3) ? eN[i] : eP[i];
    }
    __syncwarp();
    // Fluid::Fluid's Cornelius cell sizes {dt, dx, dy, dz}, src/fld.cpp:106-108
    const double dx4[4] = {dt4, g.dx, g.dy, g.dz};
    double* o = geo + (long long)k * cn::kMaxElem * kGeo;
    int n = cnw::find_surface_warp(w, dx4, e0, o);
    if (lane == 0) {
      if (n < 0) {
        atomicOr(err, ERR_SURFACE);
        n = 0;
      }
      cnt[k] = n;
    }
    __syncwarp();
  }
}

// transformToLab, src/fld.cpp:508-513
__device__ __forceinline__ void to_lab(double eta, double& vx, double& vy, double& vz) {
  const double Y = eta + 1. / 2. * log((1. + vz) / (1. - vz));
  vx = vx * cosh(Y - eta) / cosh(Y);
  vy = vy * cosh(Y - eta) / cosh(Y);
  vz = tanh(Y);
}

// pi^{mu nu} to Cartesian components at space-time rapidity eta with
// ch = cosh(eta), sh = sinh(eta), src/fld.cpp:767-786 and :1029-1048
// (index44 order)
__device__ __forceinline__ void pi_to_cartesian(double ch, double sh, const double* piC,
                                                double* pc) {
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

struct SurfArgs {
  Geo g;
  EosDev E;
  const double *Q, *Qprev, *pi, *Pi;
  double tau, dtf, ecrit, xmin, ymin, zmin;
  const int* cubes;
  const int* counters;  // [0] straddling cubes, [1] elements (device)
  int cap_cubes, cap_el;
  const double* geo;
  const int* off;
  double* rec;
  double* contrib;
};

template <int EK>
__device__ __forceinline__ void surf_element(const SurfArgs& a, int el, int ncubes);

// instantiated per EoS class, as the step's con2prim kernels are
template <int EK>
__global__ void __launch_bounds__(128) k_surf_elements(SurfArgs a) {
  const int ncubes = min(a.counters[0], a.cap_cubes), nel = min(a.counters[1], a.cap_el);
  for (int el = blockIdx.x * blockDim.x + threadIdx.x; el < nel; el += gridDim.x * blockDim.x)
    surf_element<EK>(a, el, ncubes);
}

template <int EK>
__device__ __forceinline__ void surf_element(const SurfArgs& a, int el, int ncubes) {
  // the cube whose element range holds el: the last k with off[k] <= el
  int lo = 0, hi = ncubes;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (a.off[mid] <= el)
      lo = mid;
    else
      hi = mid;
  }
  const int k = lo, e = el - a.off[k];
  const Geo& g = a.g;
  int ix, iy, iz;
  cube_cell(g, a.cubes[k], ix, iy, iz);
  const double* G = a.geo + (long long)k * cn::kMaxElem * kGeo;
  const double C[4] = {G[e * kGeo], G[e * kGeo + 1], G[e * kGeo + 2], G[e * kGeo + 3]};
  const double n0[4] = {G[4], G[5], G[6], G[7]};  // the cube's first element (src/fld.cpp:743-751)
  const double dx = g.dx, dy = g.dy, dz = g.dz, dtf = a.dtf, tau = a.tau;
  const long long N = g.N;
  const double wT[2] = {1. - C[0] / dtf, C[0] / dtf};
  const double wX[2] = {1. - C[1] / dx, C[1] / dx};
  const double wY[2] = {1. - C[2] / dy, C[2] / dy};
  const double wZ[2] = {1. - C[3] / dz, C[3] / dz};
  double QC[7] = {0., 0., 0., 0., 0., 0., 0.};
  const double* lay[2] = {a.Qprev, a.Q};
#pragma unroll 1
  for (int jt = 0; jt < 2; jt++)
#pragma unroll 1
    for (int c = 0; c < 8; c++) {
      const int jx = c >> 2, jy = (c >> 1) & 1, jz = c & 1;
      const long long i = cidx(g, ix + jx, iy + jy, iz + jz);
#pragma unroll
      for (int q = 0; q < 7; q++) QC[q] += lay[jt][q * N + i] * wT[jt] * wX[jx] * wY[jy] * wZ[jz];
    }
#pragma unroll
  for (int q = 0; q < 7; q++) QC[q] = QC[q] / (tau + C[0]);
  Prim P;
  transform_pv<EK>(a.E, QC, P);
  double TC, mubC, muqC, musC, pC;
  eos_eval_q<EK>(a.E, P.e, P.nb, TC, mubC, muqC, musC, pC);
  const double eC = P.e, nbC = P.nb;
  double vxC = P.vx, vyC = P.vy, vzC = P.vz;
  double* ct = a.contrib + (long long)el * 5;
  ct[4] = (TC > 0.4 || fabs(mubC) > 0.85) ? 1. : 0.;
  ct[0] = (eC > a.ecrit * 2.0 || eC < a.ecrit * 0.5) ? 1. : 0.;
  double piC[10], PiC = 0.;
#pragma unroll
  for (int q = 0; q < 10; q++) piC[q] = 0.;
#pragma unroll 1
  for (int c = 0; c < 8; c++) {
    const int jx = c >> 2, jy = (c >> 1) & 1, jz = c & 1;
    const long long i = cidx(g, ix + jx, iy + jy, iz + jz);
#pragma unroll
    for (int q = 0; q < 10; q++) piC[q] += a.pi[q * N + i] * wX[jx] * wY[jy] * wZ[jz];
    PiC += a.Pi[i] * wX[jx] * wY[jy] * wZ[jz];
  }
  const double v2C = vxC * vxC + vyC * vyC + vzC * vzC;
  if (v2C > 1.) {
    vxC *= sqrt(0.99 / v2C);
    vyC *= sqrt(0.99 / v2C);
    vzC *= sqrt(0.99 / v2C);
  }
  const double etaC = (a.zmin + iz * dz) + C[3];
  to_lab(etaC, vxC, vyC, vzC);
  const double gammaC = 1. / sqrt(1. - vxC * vxC - vyC * vyC - vzC * vzC);
  const double uC[4] = {gammaC, gammaC * vxC, gammaC * vyC, gammaC * vzC};
  const double tauC = tau + C[0];
  const double ch = cosh(etaC), sh = sinh(etaC);
  double ds[4];
  ds[0] = tauC * (ch * n0[0] - sh / tauC * n0[3]);
  ds[3] = tauC * (-sh * n0[0] + ch / tauC * n0[3]);
  ds[1] = tauC * n0[1];
  ds[2] = tauC * n0[2];
  double dVEff = 0.0;
#pragma unroll
  for (int q = 0; q < 4; q++) dVEff += ds[q] * uC[q];
  double pc[10];
  pi_to_cartesian(ch, sh, piC, pc);
  double dEsurfVisc = 0.;
  dEsurfVisc += pc[0] * ds[0];
  dEsurfVisc += pc[1] * ds[1];
  dEsurfVisc += pc[3] * ds[2];
  dEsurfVisc += pc[6] * ds[3];
  ct[1] = (eC + pC) * uC[0] * dVEff - pC * ds[0] + dEsurfVisc;
  ct[2] = nbC * dVEff;
  ct[3] = dVEff;
  double* r = a.rec + (long long)el * kSurfRec;
  r[0] = tau + C[0];
  r[1] = (a.xmin + ix * dx) + C[1];
  r[2] = (a.ymin + iy * dy) + C[2];
  r[3] = (a.zmin + iz * dz) + C[3];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    r[4 + q] = ds[q];
    r[8 + q] = uC[q];
  }
  r[12] = TC;
  r[13] = mubC;
  r[14] = muqC;
  r[15] = musC;
#pragma unroll
  for (int q = 0; q < 10; q++) r[16 + q] = pc[q];
  r[26] = PiC;
  r[27] = eC;
  r[28] = nbC;
}

// ===================================================================
// Corona: the element part of Fluid::outputCorona (src/fld.cpp:876-1089),
// called once at tau0.  Stages:
//   1. k_surf_energy      e at tau per corner cell (eP unused)
//   2. k_corona_flag      per interior cube: all eight corners e <= ecrit
//                         and e(corner-averaged Q / tau) >= 0.01; per-block
//                         counts
//   3. k_scan_excl        block offsets (total = element count)
//   4. k_corona_compact   element cubes in the reference's loop order
//   5. k_corona_elements  one record per element (+ its sums' contributions)
//   6. k_sum_cols         deterministic sums
// ===================================================================

// the corner-averaged Q / tau of cube (ix, iy, iz), src/fld.cpp:960-974
__device__ __forceinline__ void corona_qc(const Geo& g, const double* __restrict__ Q, int ix,
                                          int iy, int iz, double tau, double* QC) {
#pragma unroll
  for (int k = 0; k < 7; k++) QC[k] = 0.;
#pragma unroll 1
  for (int c = 0; c < 8; c++) {
    const long long i = cidx(g, ix + (c >> 2), iy + ((c >> 1) & 1), iz + (c & 1));
#pragma unroll
    for (int k = 0; k < 7; k++) QC[k] += Q[k * g.N + i] * 0.125;
  }
#pragma unroll
  for (int k = 0; k < 7; k++) QC[k] = ddivp(QC[k], tau);
}

__global__ void __launch_bounds__(kSurfBlock) k_corona_flag(Geo g, EosDev E,
                                                            const double* __restrict__ Q,
                                                            const double* __restrict__ eN,
                                                            double tau, double ecrit,
                                                            long long ncube,
                                                            unsigned char* __restrict__ flag,
                                                            int* __restrict__ blk) {
  const long long t = (long long)blockIdx.x * kSurfBlock + threadIdx.x;
  int f = 0;
  if (t < ncube) {
    int ix, iy, iz;
    cube_cell(g, t, ix, iy, iz);
    bool corona = true;
#pragma unroll
    for (int c = 0; c < 8; c++)
      if (eN[cidx(g, ix + (c >> 2), iy + ((c >> 1) & 1), iz + (c & 1))] > ecrit) corona = false;
    if (corona) {
      double QC[7];
      corona_qc(g, Q, ix, iy, iz, tau, QC);
      Prim P;
      transform_pv(E, QC, P);
      f = P.e >= 0.01;  // not the tail
    }
    flag[t] = (unsigned char)f;
  }
  const int c = __syncthreads_count(f);
  if (threadIdx.x == 0) blk[blockIdx.x] = c;
}

__global__ void __launch_bounds__(kSurfBlock) k_corona_compact(long long ncube,
                                                               const unsigned char* __restrict__ flag,
                                                               const int* __restrict__ blkoff,
                                                               int* __restrict__ cubes, int cap) {
  __shared__ int woff[kSurfBlock / 32];
  const long long t = (long long)blockIdx.x * kSurfBlock + threadIdx.x;
  const bool f = t < ncube && flag[t];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned bal = __ballot_sync(0xffffffffu, f);
  if (lane == 0) woff[w] = __popc(bal);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int k = 0; k < kSurfBlock / 32; k++) {
      const int v = woff[k];
      woff[k] = s;
      s += v;
    }
  }
  __syncthreads();
  const int slot = blkoff[blockIdx.x] + woff[w] + __popc(bal & ((1u << lane) - 1u));
  if (f && slot < cap) cubes[slot] = (int)t;  // past cap: the host grows and reruns
}

__global__ void __launch_bounds__(128) k_corona_elements(SurfArgs a) {
  const int nel = min(a.counters[0], a.cap_el);
  const Geo& g = a.g;
  const long long N = g.N;
  const double dx = g.dx, dy = g.dy, dz = g.dz, tau = a.tau;
  for (int el = blockIdx.x * blockDim.x + threadIdx.x; el < nel; el += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    cube_cell(g, a.cubes[el], ix, iy, iz);
    double QC[7];
    corona_qc(g, a.Q, ix, iy, iz, tau, QC);
    Prim P;
    transform_pv(a.E, QC, P);
    double TC, mubC, muqC, musC, pC;
    eos_eval_q(a.E, P.e, P.nb, TC, mubC, muqC, musC, pC);
    const double eC = P.e, nbC = P.nb;
    double vxC = P.vx, vyC = P.vy, vzC = P.vz;
    double* ct = a.contrib + (long long)el * 5;
    ct[0] = 0.;
    ct[4] = (TC > 0.4 || fabs(mubC) > 0.99) ? 1. : 0.;
    double piC[10], PiC = 0.;
#pragma unroll
    for (int q = 0; q < 10; q++) piC[q] = 0.;
#pragma unroll 1
    for (int c = 0; c < 8; c++) {
      const long long i = cidx(g, ix + (c >> 2), iy + ((c >> 1) & 1), iz + (c & 1));
#pragma unroll
      for (int q = 0; q < 10; q++) piC[q] += a.pi[q * N + i] * 0.125;
      PiC += a.Pi[i] * 0.125;
    }
    const double v2C = vxC * vxC + vyC * vyC + vzC * vzC;
    if (v2C > 1.) {
      vxC *= sqrt(0.99 / v2C);
      vyC *= sqrt(0.99 / v2C);
      vzC *= sqrt(0.99 / v2C);
    }
    const double etaC = (a.zmin + iz * dz) + 0.5 * dz;
    to_lab(etaC, vxC, vyC, vzC);
    const double gammaC = 1. / sqrt(1. - vxC * vxC - vyC * vyC - vzC * vzC);
    const double uC[4] = {gammaC, gammaC * vxC, gammaC * vyC, gammaC * vzC};
    const double ch = cosh(etaC), sh = sinh(etaC);
    double ds[4];
    ds[0] = tau * (ch * dx * dy * dz);
    ds[3] = tau * (-sh * dx * dy * dz);
    ds[1] = 0.0;
    ds[2] = 0.0;
    double dVEff = 0.0;
#pragma unroll
    for (int q = 0; q < 4; q++) dVEff += ds[q] * uC[q];
    double pc[10];
    pi_to_cartesian(ch, sh, piC, pc);
    double dEsurfVisc = 0.;
    dEsurfVisc += pc[0] * ds[0];
    dEsurfVisc += pc[1] * ds[1];
    dEsurfVisc += pc[3] * ds[2];
    dEsurfVisc += pc[6] * ds[3];
    ct[1] = (eC + pC) * uC[0] * dVEff - pC * ds[0] + dEsurfVisc;
    ct[2] = nbC * dVEff;
    ct[3] = dVEff;
    double* r = a.rec + (long long)el * kSurfRec;
    r[0] = tau;
    r[1] = (a.xmin + ix * dx) + 0.5 * dx;
    r[2] = (a.ymin + iy * dy) + 0.5 * dy;
    r[3] = (a.zmin + iz * dz) + 0.5 * dz;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      r[4 + q] = ds[q];
      r[8 + q] = uC[q];
    }
    r[12] = TC;
    r[13] = mubC;
    r[14] = muqC;
    r[15] = musC;
#pragma unroll
    for (int q = 0; q < 10; q++) r[16 + q] = pc[q];
    r[26] = PiC;
    r[27] = eC;
    r[28] = nbC;
  }
}

// Column sums of x[n][kSurfAcc] in a fixed tree: block partials, then one
// block over the partials in index order.
// With n_dev set, n = min(*n_dev, cap) rows are read on the device.
__global__ void __launch_bounds__(kTotBlock) k_sum_cols(const double* __restrict__ x, int n,
                                                        int ncol, double* __restrict__ out,
                                                        const int* __restrict__ n_dev, int cap) {
  __shared__ double red[kTotBlock / 32];
  if (n_dev) n = min(*n_dev, cap);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int c = 0; c < ncol; c++) {
    double s = 0.;
    for (int i = blockIdx.x * kTotBlock + threadIdx.x; i < n; i += gridDim.x * kTotBlock)
      s += x[(long long)i * ncol + c];
    s = warp_sum(s);
    if (lane == 0) red[w] = s;
    __syncthreads();
    if (w == 0) {
      double v = lane < kTotBlock / 32 ? red[lane] : 0.;
      v = warp_sum(v);
      if (lane == 0) out[blockIdx.x * ncol + c] = v;
    }
    __syncthreads();
  }
}

void launch_surf_energy(const Geo& g, const EosDev& E, const Fields& f, double tau, double taup,
                        double* eN, double* eP, cudaStream_t s) {
  const unsigned nb = (unsigned)((g.N + 127) / 128);
  if (E.kind == 5)
    k_surf_energy<EK_SMASH><<<nb, 128, 0, s>>>(g, E, f.Q, f.Qprev, tau, taup, eN, eP);
  else if (E.kind == 4)
    k_surf_energy<EK_HADRON><<<nb, 128, 0, s>>>(g, E, f.Q, f.Qprev, tau, taup, eN, eP);
  else if (E.kind == 3)
    k_surf_energy<EK_TABLE3><<<nb, 128, 0, s>>>(g, E, f.Q, f.Qprev, tau, taup, eN, eP);
  else if (E.kind == 6)
    k_surf_energy<EK_AZH><<<nb, 128, 0, s>>>(g, E, f.Q, f.Qprev, tau, taup, eN, eP);
  else if (E.kind == 7)
    k_surf_energy<EK_CMFE><<<nb, 128, 0, s>>>(g, E, f.Q, f.Qprev, tau, taup, eN, eP);
  else if (E.kind == 2)
    k_surf_energy<EK_CHIRAL><<<nb, 128, 0, s>>>(g, E, f.Q, f.Qprev, tau, taup, eN, eP);
  else
    k_surf_energy<EK_TABLE><<<nb, 128, 0, s>>>(g, E, f.Q, f.Qprev, tau, taup, eN,
                                                               eP);
}

long long surf_ncube(const Geo& g) {
  const int nix = g.nx - 4, niy = g.ny - 4, niz = g.zc1 - g.zc0;
  return (nix > 0 && niy > 0 && niz > 0) ? (long long)nix * niy * niz : 0;
}

int surf_count_blocks(const Geo& g) {
  return (int)((surf_ncube(g) + kSurfBlock - 1) / kSurfBlock);
}

void launch_surf_count(const Geo& g, const double* eN, const double* eP, double e0, int* blk,
                       int* total, cudaStream_t s) {
  const int nb = surf_count_blocks(g);
  if (nb == 0) {
    cudaMemsetAsync(total, 0, sizeof(int), s);
    return;
  }
  k_surf_count<<<nb, kSurfBlock, 0, s>>>(g, eN, eP, e0, surf_ncube(g), blk);
  k_scan_excl<<<1, kScanBlock, 0, s>>>(blk, nb, total, nullptr, 0);
}

void launch_surf_compact(const Geo& g, const double* eN, const double* eP, double e0,
                         const int* blkoff, int* cubes, int cap, cudaStream_t s) {
  const int nb = surf_count_blocks(g);
  if (nb)
    k_surf_compact<<<nb, kSurfBlock, 0, s>>>(g, eN, eP, e0, surf_ncube(g), blkoff, cubes, cap);
}

// Grid-stride launches over the device-side counts (no host round trip):
// 6 two-warp blocks per SM for Cornelius (its shared-memory limit), 8
// blocks of 128 threads per SM for the elements.
constexpr int kCornGrid = 148 * 6, kElemGrid = 148 * 8;

void launch_surf_cornelius(const Geo& g, const double* eN, const double* eP, double e0, double dtf,
                           const int* cubes, int* counters, int cap_cubes, double* geo, int* cnt,
                           unsigned* err, cudaStream_t s) {
  k_surf_cornelius<<<kCornGrid, 32 * kCornWarps, 0, s>>>(g, eN, eP, e0, dtf, cubes, counters,
                                                         cap_cubes, geo, cnt, err);
  k_scan_excl<<<1, kScanBlock, 0, s>>>(cnt, 0, counters + 1, counters, cap_cubes);
}

void launch_surf_elements(const Geo& g, const EosDev& E, const Fields& f, double tau, double dtf,
                          double ecrit, double xmin, double ymin, double zmin, const int* cubes,
                          const int* counters, int cap_cubes, int cap_el, const double* geo,
                          const int* off, double* rec, double* contrib, double* partial,
                          int npartial, cudaStream_t s) {
  SurfArgs a{g,    E,    f.Q,      f.Qprev,   f.pi,   f.Pi, tau, dtf, ecrit,  xmin, ymin, zmin,
             cubes, counters, cap_cubes, cap_el, geo, off, rec, contrib};
  if (E.kind == 5)
    k_surf_elements<EK_SMASH><<<kElemGrid, 128, 0, s>>>(a);
  else if (E.kind == 4)
    k_surf_elements<EK_HADRON><<<kElemGrid, 128, 0, s>>>(a);
  else if (E.kind == 3)
    k_surf_elements<EK_TABLE3><<<kElemGrid, 128, 0, s>>>(a);
  else if (E.kind == 6)
    k_surf_elements<EK_AZH><<<kElemGrid, 128, 0, s>>>(a);
  else if (E.kind == 7)
    k_surf_elements<EK_CMFE><<<kElemGrid, 128, 0, s>>>(a);
  else if (E.kind == 2)
    k_surf_elements<EK_CHIRAL><<<kElemGrid, 128, 0, s>>>(a);
  else
    k_surf_elements<EK_TABLE><<<kElemGrid, 128, 0, s>>>(a);
  k_sum_cols<<<npartial, kTotBlock, 0, s>>>(contrib, 0, kSurfAcc, partial, counters + 1, cap_el);
  k_sum_cols<<<1, kTotBlock, 0, s>>>(partial, npartial, kSurfAcc, partial + npartial * kSurfAcc,
                                     nullptr, 0);
}

}  // namespace vh

namespace vh {

__global__ void __launch_bounds__(32 * kCornWarps) k_cornelius_batch(
    const double* __restrict__ cubes, int n, double d0, double d1, double d2, double d3, double e0,
    int* __restrict__ counts, double* __restrict__ geo) {
  __shared__ cnw::WarpWork ws[kCornWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = blockIdx.x * kCornWarps + warp;
  if (k >= n) return;
  cnw::WarpWork& w = ws[warp];
  if (lane < 16) w.hc[lane] = cubes[(long long)k * 16 + lane];
  __syncwarp();
  const double dx4[4] = {d0, d1, d2, d3};
  const int m = cnw::find_surface_warp(w, dx4, e0, geo + (long long)k * cn::kMaxElem * kGeo);
  if (lane == 0) counts[k] = m;
}

void launch_cornelius_batch(const double* cubes, int n, const double* dx, double e0, int* counts,
                            double* geo, cudaStream_t s) {
  if (n > 0)
    k_cornelius_batch<<<(n + kCornWarps - 1) / kCornWarps, 32 * kCornWarps, 0, s>>>(
        cubes, n, dx[0], dx[1], dx[2], dx[3], e0, counts, geo);
}

void launch_corona(const Geo& g, const EosDev& E, const Fields& f, double tau, double ecrit,
                   double xmin, double ymin, double zmin, const double* eN, unsigned char* flag,
                   int* blk, int* counters, int* cubes, int cap, double* rec, double* contrib,
                   double* partial, int npartial, cudaStream_t s) {
  const int nb = surf_count_blocks(g);
  if (nb == 0) {
    cudaMemsetAsync(counters, 0, sizeof(int), s);
  } else {
    const long long ncube = surf_ncube(g);
    k_corona_flag<<<nb, kSurfBlock, 0, s>>>(g, E, f.Q, eN, tau, ecrit, ncube, flag, blk);
    k_scan_excl<<<1, kScanBlock, 0, s>>>(blk, nb, counters, nullptr, 0);
    k_corona_compact<<<nb, kSurfBlock, 0, s>>>(ncube, flag, blk, cubes, cap);
  }
  SurfArgs a{g,    E,   f.Q, f.Qprev, f.pi, f.Pi, tau, 0., ecrit, xmin, ymin, zmin,
             cubes, counters, cap, cap, nullptr, nullptr, rec, contrib};
  k_corona_elements<<<kElemGrid, 128, 0, s>>>(a);
  k_sum_cols<<<npartial, kTotBlock, 0, s>>>(contrib, 0, kSurfAcc, partial, counters, cap);
  k_sum_cols<<<1, kTotBlock, 0, s>>>(partial, npartial, kSurfAcc, partial + npartial * kSurfAcc,
                                     nullptr, 0);
}

}  // namespace vh
