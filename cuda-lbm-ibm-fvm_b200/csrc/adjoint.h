// adjoint.h -- the adjoint of the plain step on the device (adjoint.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>

#include "mg_solve.h"
#include "plain_step.h"
#include "vof_device.cuh"

namespace vof {

// 1 / ap of the Jacobi sweep for the 64 combinations of a cell's six wall
// flags (i == 1, i == nx, j == 1, j == ny, k == 1, k == nz; bit 0 .. 5).
struct InvAp {
    double v[64];
};

// One state of the step: F, u, v, w, p in the padded layout (FP32), and in
// the convergent modes the FP64 pressure the next solve starts from.
struct AdjState {
    float* f[5];
    double* p64;
};

// What the segment replay keeps of each step for the reverse pass: u*, v*,
// w* (the predictor's output) and F after the first and the second FCT sweep.
// With these, the start state and the next state (corrected velocity,
// pressure after the solve), a reversed step needs no recomputation.
struct AdjMid {
    float* f[5];
};

// Where the reverse pass takes a step's intermediates from.
enum {
    ADJ_STORE_AUTO = 0,       // kept when they fit in device memory, else recomputed
    ADJ_STORE_RECOMPUTE = 1,  // always recomputed from the step's start state
    ADJ_STORE_KEEP = 2        // always kept (allocation failure otherwise)
};

// The device side of vof_forward_record / vof_backward.  Forward: the
// context's own steps, with the state copied to a checkpoint every `every`
// steps.  Backward: per segment (last first), the segment's states are
// recomputed from its checkpoint with the engine's own buffers, then the
// steps are reversed one by one.  A reversed step needs the step's
// intermediates (u*, the pressure after the sweeps, the corrected velocity,
// F before each FCT sweep) in FP32, bit for bit the forward's values: kept by
// the replay (AdjMid, 5 fields per step of a segment) or recomputed from the
// step's start state.  The transposed kernels then run on FP64 adjoint fields.
struct AdjEngine {
    Geom g;
    int jacobi_iters;
    // convergent modes: the pressure is the solve of the mean-free system
    // (to tol), whose adjoint is the same solve on the pressure's adjoint
    int conv;
    double tol;
    int max_outer;
    MgSolver mg_fwd, mg_adj;   // forward recompute; adjoint solve
    double* p64;               // FP64 pressure of the recompute
    cudaStream_t cap;          // capture stream of the solvers' graphs
    size_t elems;           // padded elements per field
    // forward tape
    int istep0, nsteps, every, ncp;
    AdjState* cp;            // ncp checkpoints (host array of device states)
    AdjState* seg;           // every segment states (kept tapes: entries 1.. only)
    AdjMid* mid;             // kept tapes: the intermediates of every steps; else null
    int policy;              // ADJ_STORE_* for the next tape
    int keep;                // the current tape keeps the intermediates
    // the record replayed its last segment with the intermediates kept
    // (adj_record_tail): the reverse pass starts without a replay; tail_p is
    // that segment's last pressure (an engine buffer)
    bool tail_kept;
    const float* tail_p;
    // further sets of segment states and intermediates (none unless the tape
    // keeps intermediates; as many as memory allows, leaving 1/32 of the
    // device free): set i holds segment ncp - 2 - i, which the record runs
    // into it (kept[i]) as the reverse pass would replay it, so that pass
    // replays none of those segments
    static constexpr int MAX_KEPT = 64;
    int nkept;
    AdjState* kseg[MAX_KEPT];
    AdjMid* kmid[MAX_KEPT];
    bool kept[MAX_KEPT];
    size_t tape_bytes;       // device bytes of the tape
    bool recorded;
    // recompute buffers (FP32)
    PlainBuffers wb;
    CUtensorMap maps[4];
    int* status;
    float *Fin1, *Fin2, *Ftd, *A, *C, *rp, *rm;
    // adjoint fields (FP64)
    double *lF, *lu, *lv, *lw, *lp[2], *lus, *lvs, *lws, *lrhs, *lrho, *lnu;
    double *lX, *lown, *lmx, *lmn, *lpp, *lpm, *ldv, *lterm, *lLF, *lA;
    unsigned char* sel;
    int lp_cur;             // which lp buffer holds the pressure adjoint
    // plain step: lp[lp_cur] holds mu of the last transposed Jacobi stage
    // whose -N mu (the pressure adjoint) the next update applies
    bool lp_pending;
    int fct_march;          // sweep adjoints: 0 shared-memory kernels, 1 line march on large grids, 2 always march
    InvAp inv_ap;
    double* d_partial;      // block partials (body force, loss)
    int npartial;
    double* d_sums;         // [0..2] dL/dg, [3] loss
    double* h_sums;         // pinned copy
    size_t bytes;
};

// Allocate the engine for grid g (no tape yet).  Buffers are zeroed.
// mg_mode: 0 for the plain step (jacobi_iters sweeps), MG_MIXED or MG_FP64
// for the convergent solve to tol with at most max_outer V-cycles.
cudaError_t adj_create(const Geom& g, int jacobi_iters, int mg_mode, double tol, int max_outer, AdjEngine* e,
                       cudaStream_t s);
void adj_destroy(AdjEngine* e);

// (Re)allocate the tape for nsteps steps from istep0 with a checkpoint every
// `every` steps (0: ceil(sqrt(nsteps))).  e->policy decides whether the
// segment replay keeps each step's intermediates; AUTO keeps them when the
// checkpoints, segment states and intermediates leave 1/32 of the device
// memory free.
cudaError_t adj_tape(AdjEngine* e, int istep0, int nsteps, int every, cudaStream_t s);

// Copy the state x into checkpoint m.
cudaError_t adj_save(AdjEngine* e, int m, const AdjState& x, cudaStream_t s);

// First step (counted from istep0) of tape segment m, m = 0 .. ncp (ncp: the
// step count).  Segments are aligned to the end of the run: the last one holds
// `every` steps, the first one the remainder.
int adj_segment_first(const AdjEngine& e, int m);

// Whether the record may run its last segment through adj_record_tail: a tape
// that keeps intermediates, the plain pressure with an even number of sweeps
// (the pressure then ends each step in the buffer it started in).
bool adj_can_record_tail(const AdjEngine& e);

// The record's last segment, from checkpoint ncp - 1 (saved before): its steps
// run as the reverse pass replays them (intermediates and segment states
// kept, the same kernels, so the same bits), and the final state is copied to
// `out` (F, u, v, w, p) and the last step's u*, v*, w*, rhs to extra[0..3].
// The reverse pass then starts on this segment without a replay.
cudaError_t adj_record_tail(AdjEngine* e, const AdjState& out, float* const extra[4], cudaStream_t s);

// Whether the record may keep segment m (< ncp - 1) in a set of its own
// (adj_record_keep): adj_can_record_tail and a set allocated for it.
bool adj_can_keep(const AdjEngine& e, int m);

// The record's segment m, from checkpoint m (saved before), run like
// adj_record_tail into its set; the final state goes to `out`.  The record
// then saves checkpoint m + 1 from `out` and goes on with segment m + 1.
cudaError_t adj_record_keep(AdjEngine* e, int m, const AdjState& out, cudaStream_t s);

// Reverse the recorded run: L = sum over the box of F dV of the final state
// `fin`; afterwards lF, lu, lv, lw, lp[lp_cur] hold dL/d(initial state) and
// d_sums[0..3] dL/dg and L.  Waits for stream s.
cudaError_t adj_backward(AdjEngine* e, const AdjState& fin, const double box[6], double* loss, double grad_g[3],
                         cudaStream_t s);

// Kernel launches of one reversed step (recompute and adjoint).
int adj_kernels_per_step(const AdjEngine& e);

}  // namespace vof
