// jacobi_tb.h -- temporally blocked Jacobi sweeps (jacobi_tb.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "vof_device.cuh"

namespace vof {

// Largest number of sweeps one launch fuses.
constexpr int JACOBI_TB_MAX = 4;

// Tensor map (TMA descriptor) of one padded field for the sweep kernels.
cudaError_t jacobi_tb_maps(const Geom& g, const float* field, CUtensorMap* map);

// Enqueue T (1..JACOBI_TB_MAX) Jacobi sweeps reading the pressure field of
// `map_in` and the rhs of `map_rhs`, writing the interior of `pout` (a
// different buffer; its ghost cells are left as they are).  A TMA wait that
// times out sets DEV_TMA_TIMEOUT in *status.
cudaError_t jacobi_tb_launch(const Geom& g, int T, const CUtensorMap& map_in, const CUtensorMap& map_rhs,
                             float* pout, int* status, cudaStream_t s);

// One Jacobi sweep from pin (and rhs) into the interior of pout (a different
// buffer; its ghost cells are left as they are), streaming along z.
cudaError_t jacobi_col_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s);

// The same sweep with two cells per thread (scalar FP32, same bits).
cudaError_t jacobi_pairs_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s);

// The paired sweep with its wall and last planes peeled out of the march
// (unrolled VOF_JP_UNROLL times, default 2); same bits as jacobi_pairs_launch.
// down: march z downwards (the default shape only); same bits.
cudaError_t jacobi_peel_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s,
                               bool down = false);

// z chunk of a launch of bx blocks per chunk whose resident blocks number
// `wave`: the longest chunk whose last wave of blocks is 85 % full or more,
// else the one that fills it best.
int wave_kchunk(int nz, int bx, int wave);

// The paired sweep fed by bulk copies of whole rows into a shared-memory
// ring (one producer thread, bounded mbarrier waits that report
// DEV_TMA_TIMEOUT in *status); same bits as jacobi_pairs_launch.
bool jacobi_bulk_supported(const Geom& g);
cudaError_t jacobi_bulk_launch(const Geom& g, const float* pin, const float* rhs, float* pout, int* status,
                               cudaStream_t s);

// The same march with four cells per thread (16-byte loads); same bits.
cudaError_t jacobi_quad_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s);

// The paired sweep with its own column's loads copied several planes ahead
// into shared memory (cp.async); same bits as jacobi_pairs_launch.
cudaError_t jacobi_ring_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s);

// Two sweeps in one launch (the first sweep's planes kept in shared memory),
// same bits as two jacobi_pairs_launch calls; pout is a third buffer (not
// pin), whose ghost cells are left as they are.
cudaError_t jacobi_pairs2_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s);
bool jacobi_pairs2_supported(const Geom& g);

// Dynamic shared memory of one block for T fused sweeps.
size_t jacobi_tb_smem_bytes(int T);

// Raise the kernels' dynamic shared-memory ceiling (once per device).
cudaError_t jacobi_tb_configure();

}  // namespace vof
