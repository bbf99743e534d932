// mg_solve.h -- convergent pressure solve of the MIXED / FP64 modes (mg_solve.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "vof_device.cuh"

namespace vof {

enum { MG_MIXED = 1, MG_FP64 = 2 };  // inner precision: BF16 storage + FP32 math, or FP64
constexpr double MG_OMEGA = 6.0 / 7.0;  // damped-Jacobi weight (coarsest level without the dense solve)
// Smoother: Chebyshev-accelerated Jacobi of degree nu on the eigenvalues of
// D^-1 A in [MG_CHEB_HI / ratio, MG_CHEB_HI] (D^-1 A has its spectrum in [0, 2]).
constexpr double MG_CHEB_HI = 2.0;
constexpr int MG_NU_FINE = 3;           // pre/post degree on levels wider than 25 cells
constexpr double MG_RATIO_FINE = 6.0;   // eigenvalue ratio they damp (the 2x-coarsening high modes)
constexpr int MG_NU_COARSE = 8;         // pre/post degree on the small levels
constexpr double MG_RATIO_COARSE = 30.0;  // wider: these levels may coarsen by 3, 5 or 7
constexpr int MG_MAX_NU = 8;
constexpr int MG_COARSE_SWEEPS = 100;   // sweeps on a coarsest level too large for the dense solve
constexpr int MG_MAX_LEVELS = 16;
constexpr int MG_TAIL_CELLS = 4096;     // largest level that may run inside the one-block kernel
constexpr int MG_TAIL_SMEM = 200 * 1024;  // shared-memory limit of the one-block kernel
constexpr int MG_DENSE_MAX = 128;       // coarsest levels this small are solved exactly
constexpr int MG_BX = 32, MG_BY = 8;    // block of the multi-block level kernels
constexpr int MG_FLAT_THREADS = 256;    // block of the flat BF16 kernels (consecutive pairs or cells of a plane)

// One multigrid level: compact layout (i fastest, no ghosts); A e = sum over
// the non-wall neighbours of a (e_nb - e_c) with a = ax, ay, az; ratio
// (rx, ry, rz) to the next coarser level; idg[nbx*9 + nby*3 + nbz] =
// 1 / diag(A) for a cell with nbx, nby, nbz non-wall neighbours along x, y, z
// (0 where the diagonal is 0).  Smoothing step q (x_0 the start):
//   x_{q+1} = x_q + ca[q] (x_q - x_{q-1}) + cb[q] D^-1 (b - A x_q).
struct MgLevel {
    int nx, ny, nz, ncell;
    double ax, ay, az;
    double idg[27];
    double ca[MG_MAX_NU], cb[MG_MAX_NU];
    int rx, ry, rz;
    int nu;                  // pre/post smoothing degree
    int gx, gy, gz, kc;      // launch tiling: grid (gx, gy, gz) of MG_BX x MG_BY blocks, kc planes per block
    // tilings of the flat kernels (1-D blocks of MG_FLAT_THREADS, grid (x, z),
    // kc planes per block): over the cell pairs of a plane (even nx; the
    // paired smoother) and over the cells of a plane (the coarse side of the
    // paired restriction and prolongation)
    int pgx, pgz, pkc;
    int cgx, cgz, ckc;
    void* e0;                // correction, ping-pong pair
    void* e1;
    void* b;                 // right-hand side of this level
};

struct MgSolver {
    int mode;        // MG_MIXED or MG_FP64
    // MIXED: the flat paired kernels (two cells per thread, packed FP32) on
    // levels of even width and for 2x2x2 coarsening; 0: the row kernels
    // (VOF_MG_PAIRS=0)
    int pairs;
    int nlev;
    int tail;        // first level handled by the one-block kernel (nlev: none)
    int dense;       // the coarsest level is solved with the stored inverse
    int tail_smem;   // dynamic shared memory of the one-block kernel
    MgLevel lv[MG_MAX_LEVELS];
    MgLevel* d_lv;   // device copy of lv (read by the one-block kernel)
    void* d_cinv;    // dense inverse of the coarsest operator (C type), or null
    double* d_partial;  // reduction partials, 2 per block of the largest tiling
    int nblk;           // blocks of the fine tiling
    double* d_result;   // [0..1] residual sums, [2..3] sum of rhs, [4..5] sum of p, [6..7] coarse mean
    double* h_result;   // mapped pinned host copy of the residual sums (2 doubles)
    double* h_result_dev;  // its device alias
    // One outer iteration (V-cycle, p += e, new residual) captured once as a graph.
    cudaGraphExec_t iter_graph;
    const void* graph_key[3];  // rhs, p64, p32 the graph was captured with
    int graph_launches;        // kernels in it
};

struct MgStats {
    int outer;           // V-cycles done in the last solve
    double rel_initial;  // ||b - A p0|| / ||b|| at entry (warm start)
    double rel_final;    // at exit
    int launches;        // kernel launches of the last solve
};

// Level geometry of the hierarchy for grid g (no allocation); returns the level count.
int mg_plan(const Geom& g, MgLevel* lv, int max_levels);

// Plan and allocate the solver for grid g (zeroed buffers, the dense coarse
// inverse, the device level table); bytes += device bytes allocated.
// alloc_no / fail_at (optional): the caller's running count of device
// allocations and the number of the one that is to fail as if the device
// were out of memory (vof_debug_fail_alloc); the count goes on across the
// solver's own allocations.
cudaError_t mg_create(const Geom& g, int mode, MgSolver* m, cudaStream_t s, size_t* bytes, int* alloc_no = nullptr,
                      int fail_at = -1);
void mg_destroy(MgSolver* m);

// Solve A p = rhs - mean(rhs) to ||r|| <= tol ||b|| (FP64 defect correction,
// warm start from p64, gauge mean(p) = 0), then p32 = float(p64).  Each outer
// iteration is one launch of a CUDA graph (captured on `cap`, a stream of the
// same device that is not the legacy default stream, at the first call);
// waits for stream s at every outer iteration.  cudaErrorNotReady: max_outer
// reached.
cudaError_t mg_solve(const Geom& g, MgSolver& m, const float* rhs, double* p64, float* p32, double tol,
                     int max_outer, MgStats* st, cudaStream_t s, cudaStream_t cap);

// The same solve for an FP64 right-hand side (padded layout; its interior is
// read), with no FP32 copy of the solution (the adjoint of the pressure solve).
cudaError_t mg_solve64(const Geom& g, MgSolver& m, const double* rhs, double* p64, double tol, int max_outer,
                       MgStats* st, cudaStream_t s, cudaStream_t cap);

// p64 = double(p32) on the interior (after the pressure field is uploaded).
cudaError_t mg_widen(const Geom& g, const MgSolver& m, const float* p32, double* p64, cudaStream_t s);

}  // namespace vof
