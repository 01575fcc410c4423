// vh_noalloc.cu -- vh_step_noalloc: one hydro timestep on caller-owned
// device arrays, with every scratch field of the step (face fluxes, cell
// primitives, relaxation results, the updated fill fractions, the ghost-cell
// maps and the error word) carved out of one fixed, file-scope device array.
//
// Who needs it: a host code that hands this library device memory it
// already owns and cannot let a library call cudaMalloc -- for example a
// driver whose device memory is fully reserved up front by its own pool
// allocator or by another framework's caching allocator, or one that forbids
// allocation once its time loop has started.  Such a caller passes its own
// state and EoS arrays in device memory and gets a step without any device
// or host allocation.
//
// Limits and sharing: the scratch array is sized for VH_NOALLOC_MAX_CELLS
// cells (about 21 MB, held on every GPU that loads this library until the
// process exits), and every call on a device uses the same array.  Calls
// whose work overlaps on one GPU (concurrent streams or threads) race on it
// and must be serialised by the caller.  The array keeps the previous call's
// contents; the call clears the error word itself, and every other scratch
// field is fully written before it is read within one step.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/vhlle_b200.h"
#include "vh_step.cuh"

namespace {

constexpr long long kMaxCells = VH_NOALLOC_MAX_CELLS;
constexpr int kMaxDim = VH_NOALLOC_MAX_DIM;
constexpr long long kDoublesPerCell = 81;  // m2 3, Fx/Fy/Fz 21, flux 4, pA 8, pD 4,
                                           // pTh 9, pBC 9, pi0/piH0 20, Pi0/PiH0 2,
                                           // the active-cell list (ints) 1
constexpr size_t kHeaderBytes = 256 + 3 * kMaxDim * sizeof(int) + 3 * kMaxDim;  // err, maps
constexpr size_t kHeaderAligned = (kHeaderBytes + 255) / 256 * 256;
constexpr size_t kScratchBytes = kHeaderAligned + (size_t)kDoublesPerCell * kMaxCells * sizeof(double);

// The one scratch array.  In host code this name is only a stand-in for the
// symbol: its device address is obtained per device with
// cudaGetSymbolAddress below and passed to the kernels.
static __device__ __align__(256) unsigned char vh_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch[kMaxDevices] = {nullptr};

// Looks up the scratch array's device address for the current device and
// sets the step kernels' attributes, once per device.  With lazy module
// loading the look-up is also what maps the array on the device, so it
// takes device memory once: vh_noalloc_prepare does it ahead of the caller's
// pool reservation; otherwise the first vh_step_noalloc call on a device
// does it, and that first call should come before any stream capture.
cudaError_t scratch_for_current_device(unsigned char** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_setup_mutex);
  if (!g_scratch[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, vh_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if ((e = vh::step_kernels_setup()) != cudaSuccess) return e;
    g_scratch[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch[dev]);
  return cudaSuccess;
}

thread_local char g_msg[256];

vh_status nfail(vh_status st, const char* msg) {
  strncpy(g_msg, msg, sizeof g_msg - 1);
  g_msg[sizeof g_msg - 1] = 0;
  return st;
}

vh_status cfail(cudaError_t e, const char* where) {
  snprintf(g_msg, sizeof g_msg, "vh_step_noalloc: %s: %s", where, cudaGetErrorString(e));
  return VH_ERR_CUDA;
}

// Same copy sequence as the context path (src/fld.cpp:211-273).
void ghost_map_fixed(int n, int* src, unsigned char* dst) {
  for (int i = 0; i < n; i++) {
    src[i] = i;
    dst[i] = 0;
  }
  auto cl = [n](int i) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : i); };
  int s = cl(2);
  const int l[2] = {cl(1), cl(0)};
  for (int d : l) {
    src[d] = src[s];
    dst[d] = 1;
  }
  s = cl(n - 3);
  const int r[2] = {cl(n - 2), cl(n - 1)};
  for (int d : r) {
    src[d] = src[s];
    dst[d] = 1;
  }
}

}  // namespace

extern "C" const char* vh_noalloc_last_error(void) { return g_msg; }

extern "C" vh_status vh_noalloc_prepare(int device) {
  g_msg[0] = 0;
  int prev = -1;
  cudaError_t e = cudaGetDevice(&prev);
  if (e != cudaSuccess) return cfail(e, "cudaGetDevice");
  if ((e = cudaSetDevice(device)) != cudaSuccess) return cfail(e, "cudaSetDevice");
  unsigned char* base = nullptr;
  e = scratch_for_current_device(&base);
  const cudaError_t e2 = cudaSetDevice(prev);
  if (e != cudaSuccess) return cfail(e, "scratch set-up");
  if (e2 != cudaSuccess) return cfail(e2, "cudaSetDevice (restore)");
  return VH_OK;
}

extern "C" vh_status vh_step_noalloc(const vh_grid* grid, const vh_eos* eos_dev,
                                     const vh_trcoeff* tr, double tau, double dt,
                                     const vh_state_view* s, void* stream,
                                     unsigned* error_bits) {
  g_msg[0] = 0;
  if (error_bits) *error_bits = 0;
  if (!grid || !eos_dev || !tr || !s) return nfail(VH_ERR_ARG, "vh_step_noalloc: NULL argument");
  if (!s->Q || !s->Qh || !s->Qprev || !s->pi || !s->piH || !s->Pi || !s->PiH || !s->m ||
      !s->viscCorrCut)
    return nfail(VH_ERR_ARG, "vh_step_noalloc: every field of the state view is required");
  if (grid->nx < 2 || grid->ny < 2 || grid->nz < 1)
    return nfail(VH_ERR_ARG, "vh_step_noalloc: need nx >= 2, ny >= 2, nz >= 1");
  if (!(grid->xmin < grid->xmax) || !(grid->ymin < grid->ymax) || !(grid->etamin < grid->etamax))
    return nfail(VH_ERR_ARG, "vh_step_noalloc: the grid needs min < max on every axis");
  if (!(tau > 0.)) return nfail(VH_ERR_ARG, "vh_step_noalloc: tau must be positive");
  if (grid->nx > kMaxDim || grid->ny > kMaxDim || grid->nz > kMaxDim)
    return nfail(VH_ERR_ARG,
                 "vh_step_noalloc: a grid dimension exceeds VH_NOALLOC_MAX_DIM (1024)");
  const long long N = (long long)grid->nx * grid->ny * grid->nz;
  if (N > kMaxCells)
    return nfail(VH_ERR_ARG,
                 "vh_step_noalloc: grid exceeds VH_NOALLOC_MAX_CELLS (32768 cells); "
                 "use vh_create/vh_step for larger grids");
  if (eos_dev->kind == VH_EOS_TABLE3 || eos_dev->kind == VH_EOS_HADRON ||
      eos_dev->kind == VH_EOS_SMASH || eos_dev->kind == VH_EOS_AZH || eos_dev->kind == VH_EOS_CMFE)
    return nfail(VH_ERR_ARG, "vh_step_noalloc: this EoS kind needs vh_create");
  if (const char* why = vh::eos_problem(*eos_dev)) {
    snprintf(g_msg, sizeof g_msg, "vh_step_noalloc: %s", why);
    return VH_ERR_ARG;
  }
  const double dx = (grid->xmax - grid->xmin) / (grid->nx - 1);
  const double dy = (grid->ymax - grid->ymin) / (grid->ny - 1);
  if (!(dt > 0.) || dt > dx / 2. || dt > dy / 2.)
    return nfail(VH_ERR_ARG, "vh_step_noalloc: too big delta_tau (dt > dx/2 or dy/2)");

  unsigned char* base = nullptr;
  cudaError_t e = scratch_for_current_device(&base);
  if (e != cudaSuccess) return cfail(e, "scratch set-up");
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  vh::StepArgs a;
  a.g.nx = grid->nx;
  a.g.ny = grid->ny;
  a.g.nz = grid->nz;
  a.g.N = N;
  a.g.dx = dx;
  a.g.dy = dy;
  a.g.dz = grid->dz > 0. ? grid->dz : (grid->etamax - grid->etamin) / (grid->nz - 1);
  vh::geo_whole(a.g);
  a.eos.kind = eos_dev->kind;
  a.eos.conf_cnst = eos_dev->conf_cnst;
  a.eos.ne = eos_dev->ne;
  a.eos.nn = eos_dev->nn;
  a.eos.egrid = eos_dev->egrid;
  a.eos.ngrid = eos_dev->ngrid;
  a.eos.p = eos_dev->p;
  a.eos.T = eos_dev->T;
  a.eos.mub = eos_dev->mub;
  if (eos_dev->kind == VH_EOS_CHIRAL)
    for (int k = 0; k < 2; k++) {
      const vh_eos_aux& x = eos_dev->aux[k];
      a.eos.ch[k] = vh::ChiralAux{x.ne, x.nn, x.emin, x.emax, x.nmin, x.nmax, x.p, x.T, x.mub, x.mus};
    }
  a.eos.emode = a.eos.nmode = vh::GRID_BSEARCH;  // the table stays on the device
  a.eos.e0 = a.eos.einv = a.eos.n0 = a.eos.ninv = 0.f;
  a.eos.erinv = a.eos.nrinv = nullptr;  // interpolation weights by division
  a.eos.tol = 0.00001;  // src/rmn.cpp:96
  a.eos.vguess = nullptr;
  a.eos.stats = nullptr;
  a.eos.slope = 0;
  a.tr = vh::TrDev{tr->etaS0, tr->zetaS0, tr->ah, tr->al, tr->aRho, tr->T0, tr->etaSMin,
                   tr->etaSEpsilonMin, tr->etaSShiftMuB, tr->etaSScaleMuB,
                   tr->zetaSPeakEpsilon, tr->zetaSScaleBeta, tr->zetaSSigmaMinus,
                   tr->zetaSSigmaPlus, tr->etaSparam, tr->zetaSparam, tr->zetaSPeakT,
                   tr->zetaSWidthT};
  a.viscous = tr->etaS0 > 0. || tr->zetaS0 > 0. || tr->etaSparam > 0 || tr->zetaSparam > 0;

  // scratch layout: [err, clock, active count | ghost src maps | ghost dst
  // flags | pad][doubles...]
  vh::Fields& f = a.f;
  f.err = reinterpret_cast<unsigned*>(base);
  f.nactive = reinterpret_cast<int*>(base + 32);
  double* clk = reinterpret_cast<double*>(base + 16);
  a.clk = clk;
  f.gsrc = reinterpret_cast<int*>(base + 256);
  f.gdst = base + 256 + 3 * kMaxDim * sizeof(int);
  double* d = reinterpret_cast<double*>(base + kHeaderAligned);
  f.m2 = d;
  d += 3 * N;
  f.Fx = d;
  d += 7 * N;
  f.Fy = d;
  d += 7 * N;
  f.Fz = d;
  d += 7 * N;
  f.flux = d;
  d += 4 * N;
  f.pA = d;
  d += 8 * N;
  f.pD = d;
  d += 4 * N;
  f.pTh = d;
  d += 9 * N;
  f.pBC = d;
  d += 9 * N;
  f.pi0 = d;
  d += 10 * N;
  f.piH0 = d;
  d += 10 * N;
  f.Pi0 = d;
  d += N;
  f.PiH0 = d;
  d += N;
  f.active = reinterpret_cast<int*>(d);
  f.Q = s->Q;
  f.Qh = s->Qh;
  f.Qprev = s->Qprev;
  f.pi = s->pi;
  f.piH = s->piH;
  f.Pi = s->Pi;
  f.PiH = s->PiH;
  f.vcc = s->viscCorrCut;
  f.m = s->m;

  // ghost-cell maps from fixed-size host buffers (no host allocation)
  int hsrc[3 * kMaxDim];
  unsigned char hdst[3 * kMaxDim];
  ghost_map_fixed(grid->nx, hsrc, hdst);
  ghost_map_fixed(grid->ny, hsrc + grid->nx, hdst + grid->nx);
  ghost_map_fixed(grid->nz, hsrc + grid->nx + grid->ny, hdst + grid->nx + grid->ny);
  const int ng = grid->nx + grid->ny + grid->nz;
  if ((e = cudaMemcpyAsync(f.gsrc, hsrc, ng * sizeof(int), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(f.gdst, hdst, ng, cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemsetAsync(f.err, 0, sizeof(unsigned), st)))
    return cfail(e, "scratch initialisation");

  vh::launch_clock_set(clk, tau, dt, st);
  vh::launch_step(a, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return cfail(e, "kernel launch");
  // the updated fill fractions go back into the caller's array
  if ((e = cudaMemcpyAsync(f.m, f.m2, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st)))
    return cfail(e, "fill-fraction copy");
  unsigned bits = 0;
  if ((e = cudaMemcpyAsync(&bits, f.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return cfail(e, "error-word read");
  if (error_bits) *error_bits = bits;
  if (bits)
    return nfail(VH_ERR_NUMERIC, "vh_step_noalloc: numerical failure during the step "
                                 "(see error_bits)");
  return VH_OK;
}
