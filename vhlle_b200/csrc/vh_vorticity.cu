// vh_vorticity.cu -- the vorticity output of the viscous step
// (Hydro::enableVorticity, src/hdo.cpp:60-64): d_mu beta_nu with
// beta^nu = u^nu / T as ISformal stores it in every cell (src/hdo.cpp:381-611
// and 682-727) and its beta.dat interpolation at the freeze-out elements
// (src/fld.cpp:606-831).  Nothing here feeds back into the evolution.
//
// ISformal keeps ONE 4x4 matrix M for its whole cell loop (zero at the start
// of the call; loop order ix, iy, iz with iz fastest).  A cell with matter
// (e > 0 at the half-step centre) that is not next to vacuum in x/y (the
// eight-neighbour fill-fraction test) "participates": NSquant writes row 0
// of M, each row d = 1..3 whose two d-neighbours hold matter, and then adds
// a Christoffel increment to M[3][0] and M[3][3] when T > 0.  A cell next to
// vacuum writes nothing.  Every cell with matter stores M clamped to
// [-100, 100] (Cell::setDbeta, src/cll.h:173-183); an empty cell stores
// zeros (Cell::resetDbeta).  So the value of row r at a cell is the one
// written by the last participating cell at or before it that wrote row r,
// and M[3][0], M[3][3] add, in loop order, the increments of the
// participating cells after that writer.
//
// Device form, per step (six launches, off the hot step unless enabled):
//   k_vort_T            T of every cell's Qh state at tau_{n+1} (what the
//                       neighbour rows read)
//   k_vort_ops          per cell: the values NSquant writes, which rows, the
//                       two increments
//   k_vort_scan_blocks  inclusive max-scans over loop positions of the last
//   k_vort_scan_aggs    writer of each row and of the last "lone" increment
//                       (one with no row-3 write at its cell)
//   k_vort_orphan       the running M[3][0], M[3][3] at each lone increment,
//                       folded in loop order from the row-3 writer along the
//                       chain of earlier lone increments
//   k_vort_store        each cell's clamped matrix
// The additions happen in the reference's order, so every stored value is
// the reference's bit for bit.
#include <cuda_runtime.h>

#include "vh_step.cuh"
#include "vh_surface.cuh"

namespace vh {

enum : unsigned {
  VF_NONEMPTY = 1,  // e > 0 at the half-step centre (stores M, else zeros)
  VF_PART = 2,      // and not next to vacuum: NSquant writes M
  VF_SET1 = 4,      // row 1 written (x neighbours hold matter); 8: row 2, 16: row 3
  VF_SET3 = 16,
  VF_ADD = 32,      // T > 0: the Christoffel increments are added
};
constexpr int kVortBlock = 128;
constexpr int kVortScan = 512;
constexpr int kVortKeys = 5;  // rows 0..3 writers, lone increments
constexpr int kVortChain = 32;

static inline unsigned vblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

int vort_scan_blocks(long long N) { return (int)vblk(N, kVortScan); }

// loop position (ix slowest, iz fastest) <-> cell index (ix fastest)
__device__ __forceinline__ long long vort_cell(const Geo& g, long long p) {
  const long long nyz = (long long)g.ny * g.nz;
  const long long ix = p / nyz, r = p - ix * nyz;
  const long long iy = r / g.nz, iz = r - iy * g.nz;
  return ix + (long long)g.nx * (iy + (long long)g.ny * iz);
}
__device__ __forceinline__ long long vort_pos(const Geo& g, int ix, int iy, int iz) {
  return iz + (long long)g.nz * (iy + (long long)g.ny * ix);
}

// the inclusive scan value of key k at loop position p
__device__ __forceinline__ long long vort_last(const VortDev& v, long long N, int nsb, int k,
                                               long long p) {
  return max(v.last[k * N + p], v.agg[k * nsb + p / kVortScan]);
}

__device__ __forceinline__ bool vort_lone(unsigned f) {
  return (f & VF_PART) && (f & VF_ADD) && !(f & VF_SET3);
}

__device__ __forceinline__ void four_velocity(double vx, double vy, double vz, double* u) {
  u[0] = 1.0 / sqrt(1.0 - vx * vx - vy * vy - vz * vz);
  u[1] = u[0] * vx;
  u[2] = u[0] * vy;
  u[3] = u[0] * vz;
}

// T at the prims of Qh at tau_{n+1} (Cell::getPrimVarHCenter(tau) then
// EoS::eos, src/hdo.cpp:471-480): the same con2prim as k_visc_prims' pD
template <int EK>
__global__ void __launch_bounds__(kVortBlock) k_vort_T(Geo g, EosDev E,
                                                       const double* __restrict__ Qh,
                                                       const double* __restrict__ clk,
                                                       double* __restrict__ TD) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const long long N = g.N;
  const double tau = clk[0] + clk[1];
  double qs[7], q[7];
#pragma unroll
  for (int k = 0; k < 7; k++) qs[k] = Qh[k * N + i];
  q_over(qs, tau, q);
  Prim d;
  transform_pv<EK>(E, q, d, c2p_guess(E, i));
  double T, mub, p;
  eos_eval<EK>(E, d.e, d.nb, T, mub, p);
  TD[i] = T;
}

// What NSquant does to M at cell i (src/hdo.cpp:397-414, 418-459, 466-500,
// 512-546, 558-592, 606-611)
template <int EK>
__global__ void __launch_bounds__(kVortBlock) k_vort_ops(
    Geo g, EosDev E, const double* __restrict__ Q, const double* __restrict__ Qprev,
    const double* __restrict__ m, const double* __restrict__ pA, const double* __restrict__ pD,
    const double* __restrict__ pTh, const double* __restrict__ clk, VortDev v) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const long long N = g.N;
  const double dt = clk[1], tau = clk[0] + dt;
  const double eH = pA[i];  // e at the half-step centre (ISformal's test)
  if (eH <= 0.) {
    v.flag[i] = 0;
    return;
  }
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  if (maxM(m, N, cidx(g, ix + 1, iy, iz)) <= 0.9 || maxM(m, N, cidx(g, ix, iy + 1, iz)) <= 0.9 ||
      maxM(m, N, cidx(g, ix - 1, iy, iz)) <= 0.9 || maxM(m, N, cidx(g, ix, iy - 1, iz)) <= 0.9 ||
      maxM(m, N, cidx(g, ix + 1, iy + 1, iz)) <= 0.9 ||
      maxM(m, N, cidx(g, ix + 1, iy - 1, iz)) <= 0.9 ||
      maxM(m, N, cidx(g, ix - 1, iy + 1, iz)) <= 0.9 ||
      maxM(m, N, cidx(g, ix - 1, iy - 1, iz)) <= 0.9) {
    v.flag[i] = VF_NONEMPTY;  // NSquant returns before touching M
    return;
  }
  unsigned f = VF_NONEMPTY | VF_PART;
  double out[18];
  {
    // row 0: Qprev at tau - dt and Q at tau (getPrimVarPrev, getPrimVar)
    double qs[7], q[7];
    Prim P0, P1;
#pragma unroll
    for (int k = 0; k < 7; k++) qs[k] = Qprev[k * N + i];
    q_over(qs, tau - dt, q);
    transform_pv<EK>(E, q, P0, c2p_guess(E, i));
#pragma unroll
    for (int k = 0; k < 7; k++) qs[k] = Q[k * N + i];
    q_over(qs, tau, q);
    transform_pv<EK>(E, q, P1, c2p_guess(E, i));
    double T0, T1, mub, p;
    eos_eval<EK>(E, P0.e, P0.nb, T0, mub, p);
    eos_eval<EK>(E, P1.e, P1.nb, T1, mub, p);
    double u0[4], u1[4];
    four_velocity(P0.vx, P0.vy, P0.vz, u0);
    four_velocity(P1.vx, P1.vy, P1.vz, u1);
    const bool zero = eH <= 0. || P0.e <= 0. || T1 <= 0. || T0 <= 0.;
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = zero ? 0. : (u1[k] / T1 - u0[k] / T0) / dt;
  }
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
    const double e1 = pD[ip], e0 = pD[im];
    if (e1 > 0. && e0 > 0.) {
      f |= VF_SET1 << (d - 1);
      double u0[4], u1[4];
      four_velocity(pD[N + im], pD[2 * N + im], pD[3 * N + im], u0);
      four_velocity(pD[N + ip], pD[2 * N + ip], pD[3 * N + ip], u1);
      const double T1 = v.TD[ip], T0 = v.TD[im];
      const double h = d == 1 ? g.dx : d == 2 ? g.dy : g.dz * (tau + 0.5 * dt);
      const bool zero = e1 <= 0. || e0 <= 0. || T1 <= 0. || T0 <= 0.;
#pragma unroll
      for (int k = 0; k < 4; k++) out[4 * d + k] = zero ? 0. : 0.5 * (u1[k] / T1 - u0[k] / T0) / h;
    } else {
#pragma unroll
      for (int k = 0; k < 4; k++) out[4 * d + k] = 0.;
    }
  }
  const double T = pTh[i];  // T at the half-step centre (k_visc_prims)
  if (T > 0.) {
    f |= VF_ADD;
    double uH[4];
    four_velocity(pA[5 * N + i], pA[6 * N + i], pA[7 * N + i], uH);
    out[16] = uH[3] / (T * (tau - 0.5 * dt));
    out[17] = uH[0] / (T * (tau - 0.5 * dt));
  } else {
    out[16] = out[17] = 0.;
  }
#pragma unroll
  for (int k = 0; k < 18; k++) v.val[k * N + i] = out[k];
  v.flag[i] = (unsigned char)f;
}

// Block-local inclusive max-scans over loop positions of: the position if
// the cell writes row r (r = 0..3), the position if it adds a lone
// increment; -1 otherwise.  Block maxima to agg.
__global__ void __launch_bounds__(kVortScan) k_vort_scan_blocks(Geo g, VortDev v, int nsb) {
  __shared__ int wmax[kVortKeys][kVortScan / 32];
  const long long N = g.N;
  const long long p = (long long)blockIdx.x * kVortScan + threadIdx.x;
  int key[kVortKeys];
#pragma unroll
  for (int k = 0; k < kVortKeys; k++) key[k] = -1;
  if (p < N) {
    const unsigned f = v.flag[vort_cell(g, p)];
    if (f & VF_PART) {
      key[0] = (int)p;
#pragma unroll
      for (int r = 1; r <= 3; r++)
        if (f & (VF_SET1 << (r - 1))) key[r] = (int)p;
      if (vort_lone(f)) key[4] = (int)p;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kVortKeys; k++) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, key[k], o);
      if (lane >= o) key[k] = max(key[k], t);
    }
    if (lane == 31) wmax[k][warp] = key[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < kVortKeys; k++) {
      int x = lane < kVortScan / 32 ? wmax[k][lane] : -1;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, t);
      }
      if (lane < kVortScan / 32) wmax[k][lane] = x;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kVortKeys; k++) {
    if (warp > 0) key[k] = max(key[k], wmax[k][warp - 1]);
    if (p < N) v.last[k * N + p] = key[k];
    if (threadIdx.x == kVortScan - 1) v.agg[k * nsb + blockIdx.x] = key[k];
  }
}

// Exclusive max-scan of the block maxima, in place (one block).
__global__ void __launch_bounds__(1024) k_vort_scan_aggs(int* __restrict__ agg, int nsb) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  const int per = (nsb + 1023) / 1024;
  const int b = min(nsb, t * per), e = min(nsb, b + per);
  for (int k = 0; k < kVortKeys; k++) {
    int* a = agg + (long long)k * nsb;
    int mx = -1;
    for (int j = b; j < e; j++) mx = max(mx, a[j]);
    part[t] = mx;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      const int x = t >= o ? part[t - o] : -1;
      __syncthreads();
      part[t] = max(part[t], x);
      __syncthreads();
    }
    int run = t > 0 ? part[t - 1] : -1;
    for (int j = b; j < e; j++) {
      const int x = a[j];
      a[j] = run;
      run = max(run, x);
    }
    __syncthreads();
  }
}

// M[3][0], M[3][3] right after each lone increment: from the value the
// row-3 writer left (its write plus its own increment), the earlier lone
// increments after it in loop order, then this one.
__global__ void __launch_bounds__(kVortBlock) k_vort_orphan(Geo g, VortDev v, int nsb) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long N = g.N;
  if (p >= N) return;
  const long long i = vort_cell(g, p);
  if (!vort_lone(v.flag[i])) return;
  const long long L = vort_last(v, N, nsb, 3, p);  // < p: this cell writes no row 3
  double b0 = 0., b3 = 0.;                         // M starts at zero
  if (L >= 0) {
    const long long j = vort_cell(g, L);
    b0 = v.val[12 * N + j];
    b3 = v.val[15 * N + j];
    if (v.flag[j] & VF_ADD) {
      b0 = b0 + v.val[16 * N + j];
      b3 = b3 + v.val[17 * N + j];
    }
  }
  long long chain[kVortChain];
  int n = 0;
  bool walk = false;
  for (long long c = p > 0 ? vort_last(v, N, nsb, 4, p - 1) : -1; c > L;
       c = c > 0 ? vort_last(v, N, nsb, 4, c - 1) : -1) {
    if (n == min(v.chain, kVortChain)) {
      walk = true;
      break;
    }
    chain[n++] = c;
  }
  if (!walk) {
    for (int k = n - 1; k >= 0; k--) {
      const long long j = vort_cell(g, chain[k]);
      b0 = b0 + v.val[16 * N + j];
      b3 = b3 + v.val[17 * N + j];
    }
  } else {  // a long run of lone increments: visit the positions in order
    for (long long q = L + 1; q < p; q++) {
      const long long j = vort_cell(g, q);
      if (vort_lone(v.flag[j])) {
        b0 = b0 + v.val[16 * N + j];
        b3 = b3 + v.val[17 * N + j];
      }
    }
  }
  v.R[i] = b0 + v.val[16 * N + i];
  v.R[N + i] = b3 + v.val[17 * N + i];
}

__device__ __forceinline__ double clamp100(double x) {  // std::min, then std::max
  x = (100. < x) ? 100. : x;
  return (x < -100.) ? -100. : x;
}

__global__ void __launch_bounds__(kVortBlock) k_vort_store(Geo g, VortDev v, int nsb) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long N = g.N;
  if (i >= N) return;
  if (!(v.flag[i] & VF_NONEMPTY)) {
#pragma unroll
    for (int k = 0; k < 16; k++) v.dbeta[k * N + i] = 0.;
    return;
  }
  int ix, iy, iz;
  coords(g, i, ix, iy, iz);
  const long long p = vort_pos(g, ix, iy, iz);
  double o[16];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const long long L = vort_last(v, N, nsb, r, p);
    const long long j = L >= 0 ? vort_cell(g, L) : -1;
#pragma unroll
    for (int c = 0; c < 4; c++) o[4 * r + c] = j >= 0 ? v.val[(4 * r + c) * N + j] : 0.;
  }
  const long long L3 = vort_last(v, N, nsb, 3, p), Lo = vort_last(v, N, nsb, 4, p);
  if (Lo > L3) {
    const long long j = vort_cell(g, Lo);
    o[12] = v.R[j];
    o[15] = v.R[N + j];
  } else if (L3 >= 0) {
    const long long j = vort_cell(g, L3);
    if (v.flag[j] & VF_ADD) {
      o[12] = o[12] + v.val[16 * N + j];
      o[15] = o[15] + v.val[17 * N + j];
    }
  }
#pragma unroll
  for (int k = 0; k < 16; k++) v.dbeta[k * N + i] = clamp100(o[k]);
}

int launch_vorticity(const StepArgs& a, cudaStream_t s) {
  const Geo& g = a.g;
  const Fields& F = a.f;
  const VortDev& v = *a.vort;
  const unsigned nb = vblk(g.N, kVortBlock);
  const int nsb = vort_scan_blocks(g.N);
  if (a.eos.kind == 3) {  // per EoS class, as the step's con2prim kernels
    k_vort_T<EK_TABLE3><<<nb, kVortBlock, 0, s>>>(g, a.eos, F.Qh, a.clk, v.TD);
    k_vort_ops<EK_TABLE3><<<nb, kVortBlock, 0, s>>>(g, a.eos, F.Q, F.Qprev, F.m2, F.pA, F.pD,
                                                    F.pTh, a.clk, v);
  } else if (a.eos.kind == 7) {
    k_vort_T<EK_CMFE><<<nb, kVortBlock, 0, s>>>(g, a.eos, F.Qh, a.clk, v.TD);
    k_vort_ops<EK_CMFE><<<nb, kVortBlock, 0, s>>>(g, a.eos, F.Q, F.Qprev, F.m2, F.pA, F.pD,
                                                  F.pTh, a.clk, v);
  } else if (a.eos.kind == 6) {
    k_vort_T<EK_AZH><<<nb, kVortBlock, 0, s>>>(g, a.eos, F.Qh, a.clk, v.TD);
    k_vort_ops<EK_AZH><<<nb, kVortBlock, 0, s>>>(g, a.eos, F.Q, F.Qprev, F.m2, F.pA, F.pD,
                                                 F.pTh, a.clk, v);
  } else if (a.eos.kind == 2) {
    k_vort_T<EK_CHIRAL><<<nb, kVortBlock, 0, s>>>(g, a.eos, F.Qh, a.clk, v.TD);
    k_vort_ops<EK_CHIRAL><<<nb, kVortBlock, 0, s>>>(g, a.eos, F.Q, F.Qprev, F.m2, F.pA, F.pD,
                                                    F.pTh, a.clk, v);
  } else {
    k_vort_T<EK_TABLE><<<nb, kVortBlock, 0, s>>>(g, a.eos, F.Qh, a.clk, v.TD);
    k_vort_ops<EK_TABLE><<<nb, kVortBlock, 0, s>>>(g, a.eos, F.Q, F.Qprev, F.m2, F.pA, F.pD,
                                                   F.pTh, a.clk, v);
  }
  k_vort_scan_blocks<<<nsb, kVortScan, 0, s>>>(g, v, nsb);
  k_vort_scan_aggs<<<1, 1024, 0, s>>>(v.agg, nsb);
  k_vort_orphan<<<nb, kVortBlock, 0, s>>>(g, v, nsb);
  k_vort_store<<<nb, kVortBlock, 0, s>>>(g, v, nsb);
  return 6;
}

// ------------------------------------------------------------ beta.dat
// Per element: dbeta of the cube's eight cells interpolated with the
// centroid's x, y, eta weights (src/fld.cpp:641-651, 703-727), then
// d_i beta_j = J_ik J_jl dbeta_kl g_ll with the Milne-to-Cartesian Jacobian
// J = [[ch, 0, 0, -sh], [0, 1, 0, 0], [0, 0, 1, 0], [-sh, 0, 0, ch]] at the
// centroid's eta (src/fld.cpp:798-831).
__global__ void __launch_bounds__(128) k_surf_beta(Geo g, const double* __restrict__ dbeta,
                                                   double zmin, const int* __restrict__ cubes,
                                                   const int* __restrict__ counters, int cap_cubes,
                                                   int cap_el, const double* __restrict__ geo,
                                                   const int* __restrict__ off,
                                                   double* __restrict__ beta) {
  const int ncubes = min(counters[0], cap_cubes), nel = min(counters[1], cap_el);
  const long long N = g.N;
  for (int el = blockIdx.x * blockDim.x + threadIdx.x; el < nel; el += gridDim.x * blockDim.x) {
    int lo = 0, hi = ncubes;  // the cube whose element range holds el
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (off[mid] <= el)
        lo = mid;
      else
        hi = mid;
    }
    const int k = lo, e = el - off[k];
    int ix, iy, iz;
    cube_cell(g, cubes[k], ix, iy, iz);
    const double* G = geo + ((long long)k * kSurfMaxElemPerCube + e) * kSurfGeo;
    const double wX[2] = {1. - G[1] / g.dx, G[1] / g.dx};
    const double wY[2] = {1. - G[2] / g.dy, G[2] / g.dy};
    const double wZ[2] = {1. - G[3] / g.dz, G[3] / g.dz};
    double dbI[16];
#pragma unroll
    for (int q = 0; q < 16; q++) dbI[q] = 0.0;
#pragma unroll 1
    for (int c = 0; c < 8; c++) {
      const int jx = c >> 2, jy = (c >> 1) & 1, jz = c & 1;
      const long long i = cidx(g, ix + jx, iy + jy, iz + jz);
#pragma unroll
      for (int q = 0; q < 16; q++) dbI[q] += dbeta[q * N + i] * wX[jx] * wY[jy] * wZ[jz];
    }
    const double etaC = (zmin + iz * g.dz) + G[3];
    const double ch = cosh(etaC), sh = sinh(etaC);
    const double J[4][4] = {{ch, 0., 0., -sh}, {0., 1., 0., 0.}, {0., 0., 1., 0.}, {-sh, 0., 0., ch}};
    const double gl[4] = {1., -1., -1., -1.};
    double* o = beta + (long long)el * 16;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) {
        double x = 0.0;
#pragma unroll
        for (int kk = 0; kk < 4; kk++)
#pragma unroll
          for (int l = 0; l < 4; l++) x += J[a][kk] * J[b][l] * dbI[4 * kk + l] * gl[l];
        o[4 * a + b] = x;
      }
  }
}

void launch_surf_beta(const Geo& g, const double* dbeta, double zmin, const int* cubes,
                      const int* counters, int cap_cubes, int cap_el, const double* geo,
                      const int* off, double* beta, cudaStream_t s) {
  k_surf_beta<<<148 * 8, 128, 0, s>>>(g, dbeta, zmin, cubes, counters, cap_cubes, cap_el, geo,
                                      off, beta);
}

}  // namespace vh
