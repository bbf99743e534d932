// plain_step.h -- host-side interface of the FP32 drop-in step kernels.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "vof_device.cuh"

namespace vof {

// Device buffers of one context, padded layout (vof_device.cuh).
struct PlainBuffers {
    float* F;
    float* u;
    float* v;
    float* w;
    float* us;   // predictor outputs; entries outside the updated range stay 0
    float* vs;
    float* ws;
    float* rhs;  // rho/dt * div(u*)
    float* p0;   // Jacobi ping-pong pair (DeviceFields::p / ::pt)
    float* p1;
    float* p2;   // scratch pressure buffer for the blocked sweeps
    const CUtensorMap* maps;  // TMA descriptors of p0, p1, p2, rhs (in that order)
    int* status;              // device status word (DEV_* codes, tma.cuh)
    float* csf[4];            // g.csf: interface normal x, y, z and curvature per cell; else null
};

// Raise the dynamic shared-memory limit of the FCT kernels for lines of up to
// max_line interior cells.  Call once per device before the first step.
cudaError_t plain_configure(int max_line);

// Fill g->rpair / g->qpair (the density pairs of pure cells and dt over
// them) with device arithmetic.  Call once per context.
cudaError_t plain_density_pairs(Geom* g);

// Same, writing the six values through the caller's device scratch `dev6`
// on stream s (waits for the stream); allocates nothing.
cudaError_t plain_density_pairs_on(Geom* g, float* dev6, cudaStream_t s);

// True when every FCT line tile of this grid fits in shared memory.
bool plain_supported(const Geom& g);

// Kernel launches per plain step.
int plain_kernels_per_step(const Geom& g, int jacobi_iters);

// Phases of one plain step, in launch order.
enum {
    PHASE_PREDICT = 0,
    PHASE_RHS = 1,
    PHASE_JACOBI = 2,
    PHASE_CORRECT = 3,
    PHASE_SWEEP1 = 4,
    PHASE_SWEEP2 = 5,
    PHASE_SWEEP3 = 6,
    PLAIN_PHASES = 7
};

// Enqueue one plain step on stream s.  *p_parity (0/1) selects which of
// p0/p1 holds the current pressure iterate and is updated for the ping-pong.
// ev: NULL, or PLAIN_PHASES+1 events recorded around the phases.
cudaError_t plain_step(const Geom& g, const PlainBuffers& b, int istep, int jacobi_iters,
                       int* p_parity, cudaStream_t s, cudaEvent_t* ev = nullptr);

// The two halves around the pressure solve: predictor + rhs, and velocity
// correction (with pressure p) + the three FCT sweeps.  plain_step is
// plain_front, the Jacobi sweeps, plain_back.
cudaError_t plain_front(const Geom& g, const PlainBuffers& b, cudaStream_t s, cudaEvent_t* ev = nullptr);
cudaError_t plain_back(const Geom& g, const PlainBuffers& b, int istep, const float* p, cudaStream_t s,
                       cudaEvent_t* ev = nullptr);

// The pieces of plain_step: the Jacobi sweeps from the pressure in buffer
// p0/p1 selected by *p_parity (updated to the buffer holding the result), and
// the velocity correction with its boundary conditions.
cudaError_t plain_pressure(const Geom& g, const PlainBuffers& b, int jacobi_iters, int* p_parity, cudaStream_t s);
cudaError_t plain_correct(const Geom& g, const PlainBuffers& b, const float* p, cudaStream_t s);

// Kernel launches of one phase.
int plain_phase_launches(const Geom& g, int phase, int jacobi_iters);

}  // namespace vof
