// apply_bc.h -- host-side interface of the reference's apply_bc
// (voftrial1.cu:943-956) as one launch.
#pragma once
#include <cuda_runtime.h>

namespace vof {

// The six fields apply_bc sets, in its argument order; a null pointer skips
// that field.
struct BcFields {
    float* u;
    float* v;
    float* w;
    float* F;
    float* p;
    float* rho;
};

// Enqueue apply_bc on stream s for an nx x ny x nz grid with ghost cells,
// rows of px floats (px >= nx + 2) and planes of px * (ny + 2) floats.
cudaError_t apply_bc_launch(int nx, int ny, int nz, int px, const BcFields& f, cudaStream_t s);

}  // namespace vof
