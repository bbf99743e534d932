// mg_solve.h -- convergent pressure solve of the MIXED / FP64 modes (mg_solve.cu).
#pragma once
#include <cuda_runtime.h>

#include "vof_device.cuh"

namespace vof {

enum { MG_MIXED = 1, MG_FP64 = 2 };  // inner precision: BF16 storage + FP32 math, or FP64
constexpr double MG_OMEGA = 6.0 / 7.0;  // damped-Jacobi weight
constexpr int MG_NU_FINE = 2;           // pre/post sweeps on levels wider than 25 cells
constexpr int MG_NU_COARSE = 8;         // pre/post sweeps on the small levels
constexpr int MG_COARSE_SWEEPS = 100;   // sweeps on the coarsest level
constexpr int MG_MAX_LEVELS = 16;

// One multigrid level: compact layout (i fastest, no ghosts), spacing via
// ax = 1/hx^2 ..., ratio (rx, ry, rz) to the next coarser level.
struct MgLevel {
    int nx, ny, nz;
    long ncell;
    double ax, ay, az;
    int rx, ry, rz;
    void* e0;  // correction, ping-pong pair
    void* e1;
    void* b;   // right-hand side of this level
    int cur;   // which of e0/e1 holds the last result (host side)
};

struct MgSolver {
    int mode;  // MG_MIXED or MG_FP64
    int nlev;
    MgLevel lv[MG_MAX_LEVELS];
    double* d_partial;  // reduction partials
    double* d_result;   // 8 doubles
    double* h_result;   // pinned, 2 doubles
};

struct MgStats {
    int outer;           // V-cycles done in the last solve
    double rel_initial;  // ||b - A p0|| / ||b|| at entry (warm start)
    double rel_final;    // at exit
    int launches;        // kernel launches of the last solve
};

constexpr int MG_PARTIAL_DOUBLES = 2 * 296;

// Fill the level geometry of the hierarchy for grid g; returns the level count.
int mg_plan(const Geom& g, MgLevel* lv, int max_levels);

// Bytes of one stored value for the mode.
size_t mg_storage_bytes(int mode);

// Shared-memory attribute of the coarsest-level kernel (once per solver).
cudaError_t mg_configure(const MgSolver& m);

// Solve A p = rhs - mean(rhs) to ||r|| <= tol ||b|| (FP64 defect correction,
// warm start from p64, gauge mean(p) = 0), then p32 = float(p64).  Waits for
// the stream at every outer iteration.  cudaErrorNotReady: max_outer reached.
cudaError_t mg_solve(const Geom& g, MgSolver& m, const float* rhs, double* p64, float* p32, double tol,
                     int max_outer, MgStats* st, cudaStream_t s);

// p64 = double(p32) on the interior (after the pressure field is uploaded).
cudaError_t mg_widen(const Geom& g, const float* p32, double* p64, cudaStream_t s);

}  // namespace vof
