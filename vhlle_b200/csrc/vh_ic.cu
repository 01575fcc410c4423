// vh_ic.cu -- the initial state of a Monte-Carlo Glauber event built on the
// device (vh_init_glauber).
//
// The per-cell work of an IC module (the reference's IC classes end every
// cell with Cell::setPrimVar + saveQprev + setAllM, e.g.
// src/icGlauber.cpp:147-166): the participants' Gaussian-smeared density on
// the transverse grid, normalised to its maximum, times a longitudinal
// profile, cut below e_cut, and turned into tau-weighted conserved variables
// at rest.  The participants themselves (the Woods-Saxon sampling, a few
// hundred points drawn from a seeded host random stream) come from the
// caller; the smearing over every cell is what costs: 400 participants x
// 10^4 transverse cells per event.
//
//   k_ic_profile   one thread per transverse cell: the participants' sum in
//                  participant order (staged through shared memory), as the
//                  host generator adds them
//   k_ic_max       the maximum of the profile (one block)
//   k_ic_fill      every cell: e = (e_peak H[iz]) (prof / max), the cut, nb,
//                  Q, Qprev = Q, m, and the fresh-cell viscous fields
//
// exp is the correctly rounded one of vh_crmath.cuh.
#include <cuda_runtime.h>

#include <string>

#include "../../include/vhlle_b200.h"
#include "vh_crmath.cuh"
#include "vh_ctx.cuh"

namespace vh {

constexpr int kIcBlock = 128;
constexpr int kIcChunk = 512;  // participants staged per pass

__global__ void __launch_bounds__(kIcBlock) k_ic_profile(int nx, int ny, double xmin, double dx,
                                                          double ymin, double dy,
                                                          const double* __restrict__ parts,
                                                          int np, double two_s2,
                                                          double* __restrict__ prof) {
  __shared__ double sp[2 * kIcChunk];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ix = t % nx, iy = t / nx;
  const bool in = t < nx * ny;
  // Fluid::getX / getY, src/fld.h:62-63
  const double x = xmin + ix * dx, y = ymin + iy * dy;
  double sum = 0.;
  for (int base = 0; base < np; base += kIcChunk) {
    const int n = min(kIcChunk, np - base);
    __syncthreads();
    for (int k = threadIdx.x; k < 2 * n; k += blockDim.x) sp[k] = parts[2 * base + k];
    __syncthreads();
    if (in)
      for (int k = 0; k < n; k++) {
        const double ddx = x - sp[2 * k], ddy = y - sp[2 * k + 1];
        sum += crm::exp_cr(-(ddx * ddx + ddy * ddy) / two_s2);
      }
  }
  if (in) prof[t] = sum;
}

__global__ void __launch_bounds__(1024) k_ic_max(const double* __restrict__ prof, int n,
                                                 double* __restrict__ out) {
  __shared__ double s[1024];
  double m = 0.;
  for (int k = threadIdx.x; k < n; k += blockDim.x) m = fmax(m, prof[k]);
  s[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s[0];
}

__global__ void __launch_bounds__(kIcBlock) k_ic_fill(Geo g, const double* __restrict__ prof,
                                                       const double* __restrict__ pmax,
                                                       const double* __restrict__ H, double epeak,
                                                       double nbpeak, double ecut, double tau0,
                                                       Fields f) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const long long N = g.N;
  const int nxy = g.nx * g.ny;
  const int it = (int)(i % nxy), iz = (int)(i / nxy);
  const double mx = pmax[0];
  const double p = mx > 0. ? prof[it] / mx : prof[it];
  double e = (epeak * H[iz]) * p;
  if (e < ecut) e = 0.;
  const double nb = e > 0. ? (nbpeak * H[iz]) * p : 0.;
  // Cell::setPrimVar at rest (src/cll.cpp:222-241): gamma2 = 1, v2 = 0
  const double q[7] = {tau0 * e, 0., 0., 0., tau0 * nb, 0., 0.};
#pragma unroll
  for (int k = 0; k < 7; k++) {
    f.Q[k * N + i] = q[k];
    f.Qprev[k * N + i] = q[k];  // Cell::saveQprev
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
  const double mm = e > 0. ? 1. : 0.;  // Cell::setAllM
#pragma unroll
  for (int k = 0; k < 3; k++) f.m[k * N + i] = mm;
}

}  // namespace vh

extern "C" vh_status vh_init_glauber(vh_ctx* ctx, const vh_glauber_ic* ic) {
  if (!ctx || !ic || !ic->H || (ic->nparts > 0 && !ic->parts)) return VH_ERR_ARG;
  if (ic->nparts < 0 || !(ic->smear > 0.)) {
    ctx->err = "vh_init_glauber: need nparts >= 0 and smear > 0";
    return VH_ERR_ARG;
  }
  if (ctx->surf_pending) {
    ctx->err = "vh_init_glauber: a vh_surface_begin has not ended";
    return VH_ERR_STATE;
  }
  const vh::Geo& g = ctx->g;
  const int nxy = g.nx * g.ny;
  // scratch: the transverse profile, its maximum, H[nz] and the
  // participants, in the resize staging buffer (10 doubles per cell)
  const size_t need = (size_t)nxy + 1 + g.nz + 2 * (size_t)ic->nparts;
  if (need > (size_t)10 * g.N) {
    ctx->err = "vh_init_glauber: too many participants for the grid";
    return VH_ERR_ARG;
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess && !ctx->resize_tmp) {
    e = cudaMalloc(&ctx->resize_tmp, sizeof(double) * 10 * g.N);
    if (e == cudaSuccess) ctx->allocs.push_back(ctx->resize_tmp);
  }
  double* prof = ctx->resize_tmp;
  double* pmax = prof + nxy;
  double* H = pmax + 1;
  double* parts = H + g.nz;
  cudaStream_t s = ctx->stream;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(H, ic->H, sizeof(double) * g.nz, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && ic->nparts > 0)
    e = cudaMemcpyAsync(parts, ic->parts, sizeof(double) * 2 * ic->nparts,
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    const vh_grid& gr = ctx->grid;
    vh::k_ic_profile<<<(nxy + vh::kIcBlock - 1) / vh::kIcBlock, vh::kIcBlock, 0, s>>>(
        g.nx, g.ny, gr.xmin, g.dx, gr.ymin, g.dy, parts, ic->nparts,
        2 * ic->smear * ic->smear, prof);
    vh::k_ic_max<<<1, 1024, 0, s>>>(prof, nxy, pmax);
    vh::k_ic_fill<<<(unsigned)((g.N + vh::kIcBlock - 1) / vh::kIcBlock), vh::kIcBlock, 0, s>>>(
        g, prof, pmax, H, ic->epeak, ic->nb_peak, ic->ecut, ctx->tau, ctx->f);
    e = cudaGetLastError();
  }
  // the host arrays are copied before the call returns
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    ctx->err = std::string("vh_init_glauber: ") + cudaGetErrorString(e);
    return VH_ERR_CUDA;
  }
  ctx->uploaded = true;
  return VH_OK;
}
