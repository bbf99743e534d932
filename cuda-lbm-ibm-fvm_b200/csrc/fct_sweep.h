// fct_sweep.h -- one fused FCT sweep of the volume fraction (fct_sweep.cu).
#pragma once
#include <cuda_runtime.h>

#include "vof_device.cuh"

namespace vof {

// Enqueue the sweep along `axis` (0 = x, 1 = y, 2 = z) on stream s, updating F
// in place with the face velocity `vel` of that axis.  final_sweep: the last
// sweep of the step, which also applies the final clamp and the F boundary
// conditions.
cudaError_t fct_launch(const Geom& g, int axis, bool final_sweep, float* F, const float* vel, cudaStream_t s);

// The same sweep out of place: reads Fin, writes Fout (its interior cells;
// on the final sweep also every ghost cell).  On a non-final sweep Fout's
// ghost cells must already hold finite values (the next sweep reads them only
// through wall-face fluxes of zero velocity).
cudaError_t fct_launch_to(const Geom& g, int axis, bool final_sweep, const float* Fin, float* Fout, const float* vel,
                          cudaStream_t s);

// Dynamic shared memory of one sweep tile for lines of n cells.
size_t fct_smem_bytes(int axis, int n);

// Largest dynamic shared memory a tile may use.
size_t fct_smem_limit();

// Raise the kernels' dynamic shared-memory ceiling (once per device).
cudaError_t fct_configure();

}  // namespace vof
