// reduce.h -- FP64 diagnostic reductions over the step state.
#pragma once
#include <cuda_runtime.h>

#include "vof_device.cuh"

namespace vof {

// Same numbering as VOF_RED_* in include/vof.h.
enum {
    RED_VOLUME = 0,
    RED_DIV_L2 = 1,
    RED_DIV_MAX = 2,
    RED_PRES_RESID = 3,
    RED_NONFINITE = 4,
    RED_F_MIN = 5,
    RED_F_MAX = 6,
};

constexpr int RED_BLOCKS = 592;  // 4 x 148 SMs; fixed so results are bitwise reproducible

// Scratch doubles reduce_launch needs: partials of up to 3 values per block,
// then one slot whose first 4 bytes count the finished blocks of the
// single-launch field reduction (zero between launches).
constexpr int RED_SCRATCH_DOUBLES = 3 * RED_BLOCKS + 1;
// Device doubles of the result area (result slots plus the rhs mean).
constexpr int RED_RESULT_DOUBLES = 8;

struct ReduceInputs {
    const float* F;
    const float* u;
    const float* v;
    const float* w;
    const float* p;
    const float* rhs;
};

// Enqueue reduction `what`; the value lands in d_result[reduce_result_slot(what)].
// host_alias (optional): the device address of a mapped host double that
// receives the value too.  Returns in *wrote_host whether it did (the volume
// and F min / max reductions, one launch whose last block folds the partials).
cudaError_t reduce_launch(const Geom& g, const ReduceInputs& in, int what, double* d_scratch,
                          double* d_result, cudaStream_t s, double* host_alias = nullptr,
                          bool* wrote_host = nullptr);

int reduce_result_slot(int what);

}  // namespace vof
