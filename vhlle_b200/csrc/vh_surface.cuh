// vh_surface.cuh -- interior totals of Fluid::outputSurface (vh_surface.cu).
#pragma once

#include <cuda_runtime.h>

#include "vh_step.cuh"

namespace vh {

// E, Efull, Nb1, Nb2, S, Px, vt_num, vt_den, vxvy_num, vxvy_den, pi0x_num,
// pi0x_den, txxyy_num, txxyy_den, nCoreCells, nCoreCutCells (unscaled sums)
constexpr int kTotals = 16;

int totals_blocks(const Geo& g);
void launch_totals(const Geo& g, const EosDev& E, const Fields& f, double tau, double ecrit,
                   double etamin, bool viscous, double* partial, double* out, cudaStream_t s);

}  // namespace vh
