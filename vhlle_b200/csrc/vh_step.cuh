// vh_step.cuh -- internal interface between the C ABI (vh_capi.cu) and the
// step kernels (vh_step.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/vhlle_b200.h"
#include "vh_physics.cuh"

namespace vh {

struct Geo {
  int nx, ny, nz;
  long long N;
  double dx, dy, dz;
  // the freeze-out surface's and the totals' window in eta (vh_set_slab):
  // hypercubes whose lowest corner plane is in [zc0, zc1), interior cells
  // in [zt0, zt1), and where these planes sit in the whole grid (plane 0 is
  // plane zoff of nzg); the whole grid by default ([2, nz - 2), 0, nz)
  int zc0, zc1, zt0, zt1, zoff, nzg;
};

// the default window of a whole grid
inline void geo_whole(Geo& g) {
  g.zc0 = g.zt0 = 2;
  g.zc1 = g.zt1 = g.nz - 2;
  g.zoff = 0;
  g.nzg = g.nz;
}

// Fluid::getCell index with clamping (src/fld.h:70-78)
__device__ __forceinline__ long long cidx(const Geo& g, int ix, int iy, int iz) {
  ix = ix > 0 ? ix : 0;
  ix = ix < g.nx ? ix : g.nx - 1;
  iy = iy > 0 ? iy : 0;
  iy = iy < g.ny ? iy : g.ny - 1;
  iz = iz > 0 ? iz : 0;
  iz = iz < g.nz ? iz : g.nz - 1;
  return (long long)ix + (long long)g.nx * iy + (long long)g.nx * g.ny * iz;
}

__device__ __forceinline__ void coords(const Geo& g, long long i, int& ix, int& iy, int& iz) {
  ix = (int)(i % g.nx);
  const long long r = i / g.nx;
  iy = (int)(r % g.ny);
  iz = (int)(r / g.ny);
}

__device__ __forceinline__ double maxM(const double* __restrict__ m, long long N, long long i) {
  return smax(m[i], smax(m[N + i], m[2 * N + i]));
}

// Device pointers of every field the step touches (component-major).
struct Fields {
  double *Q, *Qh, *Qprev;        // [7][N]
  double *pi, *piH;              // [10][N]
  double *Pi, *PiH, *vcc;        // [N]
  double *m, *m2;                // [3][N] fill fractions (double-buffered)
  double *Fx, *Fy, *Fz;          // [7][N] face fluxes on the +dir side
  double *flux;                  // [4][N] viscous flux accumulator
  double *pA;                    // [8][N] prims of Qh at tau_{n+1} - dt/2
  double *pD;                    // [4][N] e, v of Qh at tau_{n+1}
  double *pTh;                   // [9][N] thermodynamics and transport at pA
  double *pBC;                   // [9][N] four-velocities for NSquant's d/dtau
  double *pi0, *piH0;            // [10][N] IS relaxation results
  double *Pi0, *PiH0;            // [N]
  int *active, *nactive;         // [N] cells with matter (e > 0) for the
                                 // relaxation, and their count ([1])
  int *gsrc;                     // [nx+ny+nz] ghost-cell source map
  unsigned char *gdst;           // [nx+ny+nz] ghost-cell destination flags
  unsigned *err;                 // device error word
};

// Device buffers of the vorticity output (Hydro::enableVorticity).
struct VortDev {
  double* dbeta;        // [16][N] d_mu beta_nu per cell (4 mu + nu), clamped
  double* TD;           // [N] T at the prims of Qh at tau_{n+1}
  double* val;          // [18][N] the 16 values NSquant writes, the 2 increments
  double* R;            // [2][N] running M[3][0], M[3][3] at lone increments
  unsigned char* flag;  // [N] VF_* bits
  int* last;            // [5][N] per loop position: last writer positions
  int* agg;             // [5][blocks] block maxima, then their prefixes
  int chain = 32;       // lone increments followed back before the ordered walk
};
int vort_scan_blocks(long long N);

struct StepArgs {
  Geo g;
  EosDev eos;
  TrDev tr;
  Fields f;
  const double* clk;  // device [tau, dt] of the step (launch_clock_set)
  bool viscous;
  int block = 128;    // threads per block of the step kernels (64 or 128; the
                      // relaxation kernel always uses 128)
  const VortDev* vort = nullptr;  // vorticity on (viscous steps only)
};

// A batch's stage-batched step (vh_batch.cu): one launch per stage over
// the blocks of every event.  StepDev is one event's step arguments in
// device memory (f.m the current fill fractions, f.m2 the updated ones, as
// launch_step leaves them); a work item is one block of one event.
struct StepDev {
  Geo g;
  EosDev eos;
  TrDev tr;
  Fields f;
  double* clk;
  int viscous;
};
struct BItem {
  int ev;   // index into the StepDev array
  int blk;  // block of that event's grid (128 cells each)
};
constexpr int kBatchBlock = 128;

// The EoS class instantiation launch_step picks for an EoS descriptor.
int step_ek(const EosDev& E);
// One step of nev events (evs: device), work items covering every event's
// nblk(N, kBatchBlock) blocks (items: device); every event with EoS class
// ek and the same viscous flag.  Returns the number of launches.
int launch_step_batched(int ek, bool viscous, const StepDev* evs, int nev, const BItem* items,
                        int nitems, cudaStream_t s);
// launch_clock_op on the clocks of nev events at once (ns: device, each
// event's n for ops 1 and 2)
void launch_clock_op_batched(const StepDev* evs, int nev, int op, const int* ns, cudaStream_t s);

// ISformal's dbeta for every cell (after k_visc_prims, before the viscous
// update changes Q); returns the number of launches
int launch_vorticity(const StepArgs& a, cudaStream_t s);

// Kernel kinds, for per-kernel timing.
enum KernelKind {
  KK_UPDATE_M = 0, KK_FACE_X, KK_FACE_Y, KK_FACE_Z, KK_UPDATE, KK_GHOST, KK_VISC_PRIMS,
  KK_IS_RELAX, KK_IS_ADVECT, KK_VISC_UPDATE, KK_VORT, KK_COUNT
};
extern const char* const kKernelNames[KK_COUNT];

// Called after each launch with its kind (used to record timing events).
struct LaunchMarker {
  virtual void after(int kind) = 0;
  virtual ~LaunchMarker() {}
};

// Function attributes the step kernels need (the relaxation's 55 KB of
// dynamic shared memory), on the current device; before the first launch
// there and outside any stream capture.
cudaError_t step_kernels_setup();

// Enqueues one performStep on stream s; returns the number of launches.
// Leaves the updated fill fractions in f.m2 (the caller swaps m and m2).
int launch_step(const StepArgs& a, cudaStream_t s, LaunchMarker* mk = nullptr);
void launch_clock_set(double* clk, double tau, double dt, cudaStream_t s);
// op 0: tau += dt; 1: dt = dt / n; 2: dt = dt * n
void launch_clock_op(double* clk, int op, int n, cudaStream_t s);
// gathers ncomp planes of the x2 resized grid from src into dst
void launch_resize_gather(const Geo& g, const double* src, double* dst, int ncomp,
                          cudaStream_t s);
// Up to nine fields (pointer, components) for launch_planes.
struct PlaneFields {
  double* p[9];
  int ncomp[9];
  int nfield, ncomp_total;
};
// z-planes [z0, z0 + nz) of every field to (pack) or from a contiguous
// buffer [field][component][plane][nx*ny]
void launch_planes(const PlaneFields& pf, long long N, long long nxy, int z0, int nz,
                   double* buf, bool pack, cudaStream_t s);

void launch_transform_pv(const EosDev& E, const double* Q, long long n, double* out,
                         cudaStream_t s);
void launch_eos_eval(const EosDev& E, const double* e, const double* nb, long long n, double* out,
                     cudaStream_t s);
void launch_transport(const TrDev& tr, const double* in, long long n, double* out,
                      cudaStream_t s);

// What is wrong with an EoS descriptor the device cannot evaluate (unknown
// kind, a table smaller than 2 x 2 or larger than 2^30 points, missing
// arrays, a chiral table whose range is empty or not finite), or NULL.
// Shared by vh_create and vh_step_noalloc (vh_capi.cu).
const char* eos_problem(const vh_eos& e);

}  // namespace vh
