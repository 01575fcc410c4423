// vh_surface.cuh -- interior totals of Fluid::outputSurface (vh_surface.cu).
#pragma once

#include <cuda_runtime.h>

#include "vh_step.cuh"

namespace vh {

// E, Efull, Nb1, Nb2, S, Px, vt_num, vt_den, vxvy_num, vxvy_den, pi0x_num,
// pi0x_den, txxyy_num, txxyy_den, nCoreCells, nCoreCutCells (unscaled sums)
constexpr int kTotals = 16;

// freeze-out element record: tau, x, y, eta, dSigma[4], u[4], T, muB, muQ,
// muS, pi_cart[10] (index44 order), Pi, e, nb
constexpr int kSurfRec = 29;
// per-element contributions: nsusp, EtotSurf, nbSurf, vEff, high-T/muB flag
constexpr int kSurfAcc = 5;
constexpr int kSurfMaxElemPerCube = 10;
constexpr int kSurfGeo = 8;

// interior cube t (loop order, iz fastest) -> its lowest corner cell; in
// eta the cubes of the window [zc0, zc1)
__device__ __forceinline__ void cube_cell(const Geo& g, long long t, int& ix, int& iy, int& iz) {
  const int niz = g.zc1 - g.zc0, niy = g.ny - 4;
  iz = g.zc0 + (int)(t % niz);
  iy = 2 + (int)((t / niz) % niy);
  ix = 2 + (int)(t / ((long long)niz * niy));
}

int totals_blocks(const Geo& g);
void launch_totals(const Geo& g, const EosDev& E, const Fields& f, double tau, double ecrit,
                   double etamin, bool viscous, double* partial, double* out, cudaStream_t s);

long long surf_ncube(const Geo& g);
int surf_count_blocks(const Geo& g);
void launch_surf_energy(const Geo& g, const EosDev& E, const Fields& f, double tau, double taup,
                        double* eN, double* eP, cudaStream_t s);
// per-block counts into blk[], exclusive offsets in place, the sum to *total
void launch_surf_count(const Geo& g, const double* eN, const double* eP, double e0, int* blk,
                       int* total, cudaStream_t s);
// the first min(count, cap) straddling cubes in loop order
void launch_surf_compact(const Geo& g, const double* eN, const double* eP, double e0,
                         const int* blkoff, int* cubes, int cap, cudaStream_t s);
// Cornelius on the counters[0] (at most cap_cubes) listed cubes; cnt[]
// becomes the element offsets and counters[1] the element total
void launch_surf_cornelius(const Geo& g, const double* eN, const double* eP, double e0, double dtf,
                           const int* cubes, int* counters, int cap_cubes, double* geo, int* cnt,
                           unsigned* err, cudaStream_t s);
// records and per-element sums of the counters[1] (at most cap_el) elements;
// the sums land in partial[npartial*kSurfAcc ..]
void launch_surf_elements(const Geo& g, const EosDev& E, const Fields& f, double tau, double dtf,
                          double ecrit, double xmin, double ymin, double zmin, const int* cubes,
                          const int* counters, int cap_cubes, int cap_el, const double* geo,
                          const int* off, double* rec, double* contrib, double* partial,
                          int npartial, cudaStream_t s);

// Fluid::outputCorona's elements (eN from launch_surf_energy at tau):
// counters[0] = the element count; the first min(count, cap) records and
// contributions are written, their sums land in partial[npartial*kSurfAcc ..]
void launch_corona(const Geo& g, const EosDev& E, const Fields& f, double tau, double ecrit,
                   double xmin, double ymin, double zmin, const double* eN, unsigned char* flag,
                   int* blk, int* counters, int* cubes, int cap, double* rec, double* contrib,
                   double* partial, int npartial, cudaStream_t s);

// beta.dat's 16 Cartesian d_mu beta_nu of each element of the last
// launch_surf_elements call (same cubes, counters, geo and offsets), from
// the cells' dbeta[16][N], into beta[cap_el][16]
void launch_surf_beta(const Geo& g, const double* dbeta, double zmin, const int* cubes,
                      const int* counters, int cap_cubes, int cap_el, const double* geo,
                      const int* off, double* beta, cudaStream_t s);

// Cornelius on n independent hypercubes (16 corner values each): counts[k]
// elements (-1 where the reference stops), geo[k][10][8] centroid + normal
void launch_cornelius_batch(const double* cubes, int n, const double* dx, double e0, int* counts,
                            double* geo, cudaStream_t s);

}  // namespace vh
