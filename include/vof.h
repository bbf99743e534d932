/*
 * vof.h -- C-ABI of the B200 two-phase VOF step library (libvof_b200.so).
 *
 * The library replaces the time-loop body of voftrial1.cu
 * (voftrial1.cu:1361-1401): rho/nu from the volume fraction, the explicit
 * momentum predictor, the Jacobi pressure sweeps, the velocity correction,
 * the free-slip velocity boundary conditions, the three directionally split
 * FCT sweeps of the volume fraction in the istep-dependent order, the final
 * clamp and the zero-gradient volume-fraction boundary conditions.
 *
 * Conventions (they differ from the reference's host launchers on purpose):
 *  - Every entry point returns an int status: VOF_OK (0) or a negative
 *    VOF_E_* code.  The library never calls exit().  The CUDA error behind a
 *    VOF_E_CUDA is kept and returned by vof_last_cuda_error().
 *  - All work is enqueued on the stream given to vof_create (a cudaStream_t
 *    passed as void*; NULL means the legacy default stream, which is what the
 *    reference uses).  vof_step and vof_run do not synchronise the host.
 *  - One context per host thread.  Fields cross the boundary in the
 *    reference's own layout: (nx+2)(ny+2)(nz+2) floats, i fastest, one ghost
 *    layer (voftrial1.cu:66-70); the context keeps a padded copy internally.
 */
#ifndef VOF_B200_H
#define VOF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VOF_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
#define VOF_OK               0
#define VOF_E_INVALID      (-1)  /* bad argument (null pointer, bad field id, ...) */
#define VOF_E_SIZE         (-2)  /* grid size out of the supported range         */
#define VOF_E_NOMEM        (-3)  /* device or pinned host allocation failed        */
#define VOF_E_CUDA         (-4)  /* a CUDA runtime call failed                     */
#define VOF_E_NOT_CONVERGED (-5) /* iterative solve hit its iteration cap          */
#define VOF_E_NONFINITE    (-6)  /* watchdog found NaN/Inf in the state            */
#define VOF_E_STATE        (-7)  /* call not valid in the current context state    */
#define VOF_E_UNSUPPORTED  (-8)  /* feature not built / mode not available         */
#define VOF_E_TIMEOUT      (-9)  /* a bounded device-side wait ran out (reported by vof_sync) */

/* ---- solver modes ------------------------------------------------------ */
#define VOF_MODE_PLAIN  0   /* FP32, jacobi_iters Jacobi sweeps: the drop-in path */
#define VOF_MODE_MIXED  1   /* FP64 defect correction over a BF16-stored/FP32 inner solve */
#define VOF_MODE_FP64   2   /* same convergent projection, every field in FP64    */

/* ---- field identifiers (vof_upload / vof_download) --------------------- */
#define VOF_FIELD_F      0  /* volume fraction (DeviceFields::F)      */
#define VOF_FIELD_U      1  /* x face velocity, u[i] on face i-1/2    */
#define VOF_FIELD_V      2
#define VOF_FIELD_W      3
#define VOF_FIELD_P      4  /* pressure (current Jacobi iterate)      */
#define VOF_FIELD_USTAR  5  /* predictor output of the last step      */
#define VOF_FIELD_VSTAR  6
#define VOF_FIELD_WSTAR  7
#define VOF_FIELD_RHS    8  /* rho/dt * div(u*) of the last step (no reference buffer) */
#define VOF_NUM_FIELDS   9

/* ---- reductions (vof_reduce) -------------------------------------------- */
#define VOF_RED_VOLUME      0  /* sum over interior cells of F*dx*dy*dz (FP64)         */
#define VOF_RED_DIV_L2      1  /* sqrt(sum of (div u)^2) over interior cells (FP64)    */
#define VOF_RED_DIV_MAX     2  /* max |div u| over interior cells                      */
#define VOF_RED_PRES_RESID  3  /* ||b - A p|| / ||b|| of the last pressure system,
                                  b = rhs with its mean removed (FP64)                 */
#define VOF_RED_NONFINITE   4  /* number of NaN/Inf values in F,u,v,w,p (as a double)  */
#define VOF_RED_F_MIN       5  /* min of F over interior cells                         */
#define VOF_RED_F_MAX       6  /* max of F over interior cells                         */
#define VOF_NUM_REDUCTIONS  7

/*
 * Mirrors struct Params (voftrial1.cu:27-41) field for field and in the same
 * order, followed by the additions this library needs.
 */
typedef struct vof_params {
    int nx, ny, nz;
    int imin, imax;
    int jmin, jmax;
    int kmin, kmax;
    float Lx, Ly, Lz;
    float rho_l, rho_g;
    float nu_l, nu_g;
    float sigma;            /* stored and reported; read only by the optional surface-tension
                               term (surface_tension = 1; the reference's kernels never read it) */
    float gx, gy, gz;
    float dt;
    float dx, dy, dz;
    float dxi, dyi, dzi;
    int nTot;
    /* ---- additions (no counterpart in Params) ---- */
    int jacobi_iters;       /* plain mode: sweeps per step; voftrial1.cu:1371 hardcodes 10 */
    int mode;               /* VOF_MODE_*                                                   */
    int inner_sweeps;       /* reserved (kept for the ABI layout): the multigrid inner solve of the
                               mixed/fp64 modes uses fixed Chebyshev smoothing degrees (3 on levels
                               wider than 25 cells, 8 below); vof_params_init sets 32, unused */
    int max_outer;          /* mixed/fp64 modes: cap on defect-correction iterations        */
    double tol;             /* mixed/fp64 modes: target ||b-Ap||/||b|| (default 1e-8)       */
    int surface_tension;    /* 1: add the continuum-surface-force acceleration sigma kappa
                               grad(F) / rho to u*, v*, w* after the predictor (an extension:
                               the reference has no surface tension, so 1 departs from it);
                               0 (default): the reference's step                             */
} vof_params;

typedef struct vof_ctx vof_ctx;

/* Library ABI version (VOF_ABI_VERSION of the build). */
int vof_abi_version(void);

/* Short static description of a status code. */
const char* vof_error_string(int status);

/*
 * Fill *p for an nx x ny x nz grid the way voftrial1.cu:1262-1291 fills
 * cpar_host (same float expressions for dx and dxi), with the reference's
 * constants: 0.1 m box, rho 1000/50, nu 1e-6/1.5e-5, sigma 0.007,
 * g = (0,-5,0), dt 4e-6, plus jacobi_iters = 10 and mode = VOF_MODE_PLAIN.
 * Callers change gx/gy/gz, dt, ... afterwards and call vof_params_finalize.
 */
int vof_params_init(vof_params* p, int nx, int ny, int nz);

/*
 * Recompute the derived members (imin..kmax, dx..dzi, nTot) from nx,ny,nz
 * and Lx,Ly,Lz with the reference's float expressions (voftrial1.cu:1268-1291).
 */
int vof_params_finalize(vof_params* p);

/*
 * Create a context: validates *p, allocates every device buffer zero-filled
 * (voftrial1.cu:1200-1203, 1306-1326) in the padded internal layout.
 * `stream` is a cudaStream_t (NULL = legacy default stream).
 * Replaces: DeviceFields + alloc_field + cudaMemcpyToSymbol(cpar)
 * (voftrial1.cu:1176-1203, :1293, :1303-1326).
 */
int vof_create(const vof_params* p, void* stream, vof_ctx** out);

/* Release every buffer of the context (voftrial1.cu:1205-1226). NULL is a no-op. */
void vof_destroy(vof_ctx* ctx);

/* Copy of the parameters the context runs with. */
int vof_get_params(const vof_ctx* ctx, vof_params* out);

/*
 * Copy one field from `src` (reference layout, nTot floats) into the context.
 * src_is_device != 0: src is a device pointer; otherwise host memory (pinned
 * or pageable).  Stream-ordered; host memory must stay valid until the
 * stream reaches the copy (vof_sync).
 */
int vof_upload(vof_ctx* ctx, int field, const float* src, int src_is_device);

/* Copy one field out of the context into `dst` (reference layout, nTot floats). */
int vof_download(vof_ctx* ctx, int field, float* dst, int dst_is_device);

/*
 * Planes k0 .. k0+nk-1 (0 <= k0, k0+nk <= nz+2; ghost planes included) of
 * one field, in the reference layout of a plane ((ny+2)(nx+2) floats, i
 * fastest, planes consecutive), out of or into the context.  The halo
 * exchange of a z-slab decomposition moves planes with these (no counterpart
 * in the reference, which runs on one GPU; the host loop it would sit in is
 * voftrial1.cu:1361-1401).  Device buffers: stream-ordered, no host
 * synchronisation; host buffers: vof_get_planes waits for the copy,
 * vof_put_planes needs the host memory valid until the stream reaches the
 * copy.  vof_put_planes of VOF_FIELD_P: VOF_E_UNSUPPORTED in the convergent
 * modes (their pressure state is the FP64 copy).
 */
int vof_get_planes(vof_ctx* ctx, int field, int k0, int nk, float* dst, int dst_is_device);
int vof_put_planes(vof_ctx* ctx, int field, int k0, int nk, const float* src, int src_is_device);

/*
 * One time step, exactly the sequence of voftrial1.cu:1364-1401 for the
 * given istep (the value the reference's loop has after `++istep`, so the
 * first step is istep = 1; istep % 3 picks the FCT sweep order,
 * voftrial1.cu:1384-1396).
 */
int vof_step(vof_ctx* ctx, int istep);

/*
 * Steps istep0 .. istep0+nsteps-1 through captured CUDA graphs (one per
 * sweep order and Jacobi-buffer parity).  Same results as nsteps vof_step calls.
 */
int vof_run(vof_ctx* ctx, int istep0, int nsteps);

/*
 * Per-phase timing (no reference counterpart; voftrial1.cu times only the
 * whole loop, voftrial1.cu:1359, 1416-1420).  Runs one vof_step with CUDA
 * events recorded on the context's stream around each phase, waits for it,
 * and writes the milliseconds of phase q to phase_ms[q] and its kernel
 * launches to launches[q] (either may be NULL) for q < min(nphase,
 * VOF_PHASES).  Phases: predict, rhs, jacobi, correct, sweep1, sweep2, sweep3.
 */
#define VOF_PHASES 7
int vof_step_timed(vof_ctx* ctx, int istep, float* phase_ms, int* launches, int nphase);

/* Name of phase q of vof_step_timed ("predict", "jacobi", ...), NULL if out of range. */
const char* vof_phase_name(int phase);

/*
 * Wait for all work enqueued on the context's stream.  Also reports
 * VOF_E_TIMEOUT if a kernel's bounded wait on an asynchronous copy ran out
 * since the last call (the state is then invalid).
 */
int vof_sync(vof_ctx* ctx);

/* Blocking reduction over the current state (VOF_RED_*); result in *out. */
int vof_reduce(vof_ctx* ctx, int what, double* out);

/*
 * vof_reduce over the interior cells of planes k0..k1 only (1 <= k0 <= k1 <=
 * nz), for VOF_RED_VOLUME, F_MIN, F_MAX, DIV_L2 and DIV_MAX (a plane's
 * divergence uses the w faces above it); VOF_E_UNSUPPORTED for the others.
 * The ranks of a z-slab decomposition reduce over the planes they own and
 * combine (volumes add, DIV_L2 as the root of the summed squares).
 */
int vof_reduce_range(vof_ctx* ctx, int what, int k0, int k1, double* out);

/*
 * vof_reduce_range, stream-ordered like vof_reduce_async: *host_out receives
 * the value when the stream gets there (mapped pinned memory is written by the
 * reduction kernel itself), and the host must vof_sync before reading it.  A
 * slab rank reads its partial volume every step with no host synchronisation.
 */
int vof_reduce_range_async(vof_ctx* ctx, int what, int k0, int k1, double* host_out);

/*
 * Stream-ordered reduction: the result is written to *host_out (which should
 * be pinned host memory) when the stream reaches this point; the host must
 * vof_sync before reading it.  No host synchronisation inside.  For pinned
 * memory mapped into the device (cudaHostAlloc / cudaHostRegister on a 64-bit
 * system) the volume and F min / max reductions are one kernel that writes
 * *host_out itself; otherwise a copy follows the kernels.
 */
int vof_reduce_async(vof_ctx* ctx, int what, double* host_out);

/*
 * One plain step with no allocation at all (no counterpart in the reference).
 * For callers that must not allocate device memory while they step: programs
 * whose GPU memory is owned up front by their own pool or allocator, or loops
 * that cannot afford cudaMalloc's device-wide synchronisation and latency.
 * The caller owns F, u, v, w, p as device buffers in the reference layout
 * (nTot floats each) and they are updated in place, with results identical to
 * a fresh context doing vof_upload + vof_step(istep) + vof_download.
 * Scratch lives in a fixed device array of VOF_NOALLOC_ARENA_FLOATS floats
 * (8 MiB, held by every GPU that loads the library until exit) that must hold
 * 11 padded fields of round_up(nx+2, 32) * (ny+2) * (nz+2) floats: grids up
 * to about 48^3 fit; larger ones return VOF_E_SIZE without doing anything.
 * The first call on a device looks up the array's device address (with that
 * device current); make that first call before any stream capture.  All calls
 * share the array (each clears what it uses first), so calls that overlap on
 * the GPU race.  The call waits for `stream` before returning.  Only
 * VOF_MODE_PLAIN.  On VOF_E_TIMEOUT (a bounded device-side wait ran out) the
 * caller's buffers are left as they were passed in.
 */
#define VOF_NOALLOC_ARENA_FLOATS (2u << 20)
int vof_step_noalloc(const vof_params* p, float* F, float* u, float* v, float* w, float* pres, int istep,
                     void* stream);

/* ---- boundary conditions ------------------------------------------------ */
/*
 * The reference's apply_bc (voftrial1.cu:943-956: set_bc_j_kernel,
 * set_bc_i_kernel, set_bc_k_kernel of :105-228, in that order), as one
 * stream-ordered launch with the same result.  Ghost cells of F, p (and rho)
 * copy the nearest interior cell, edges and corners included.  The
 * wall-normal velocity is zeroed on the first and last faces (u at i = imin
 * and imax+1, v at j = jmin and jmax+1, w at k = kmin and kmax+1).  The other
 * velocity components' ghosts copy the neighbouring row as the three passes
 * leave them.  The reference's time loop never calls apply_bc; these calls
 * are for callers that do.
 *
 * vof_apply_bc: on the context's current state (F, u, v, w, p; rho is never
 * stored).  VOF_E_UNSUPPORTED in the convergent modes, where the pressure
 * state is its FP64 copy.
 */
int vof_apply_bc(vof_ctx* ctx);

/*
 * vof_apply_bc_fields: apply_bc's own signature, on caller-owned device
 * buffers in the reference layout (p->nTot floats each).  A NULL pointer
 * skips that field.  Enqueued on `stream` (NULL: the legacy default stream,
 * as the reference launches); no host synchronisation.  VOF_E_SIZE for an
 * empty or oversized grid, VOF_E_INVALID for inconsistent parameters.
 */
int vof_apply_bc_fields(const vof_params* p, float* u, float* v, float* w, float* F, float* pres, float* rho,
                        void* stream);

/*
 * Convergent modes (VOF_MODE_MIXED, VOF_MODE_FP64; no counterpart in the
 * reference): V-cycles done by the last pressure solve and its relative
 * residual ||b - A p|| / ||b|| (FP64, b = rhs - mean) at entry and at exit.
 * VOF_E_STATE in VOF_MODE_PLAIN.
 */
int vof_solver_stats(const vof_ctx* ctx, int* outer, double* rel_initial, double* rel_final);

/* ---- adjoint (extension; the reference has no adjoint) ----------------------
 * Gradient of L = sum of F dV over the interior cells whose centre lies
 * strictly inside box = {x0, x1, y0, y1, z0, z1} after a recorded run, with
 * respect to the run's initial state and the body force.  Derivative
 * conventions at the step's non-smooth points: a branch (upwinding, the FCT
 * flux direction) differentiates the side the forward took, fmaxf / fminf the
 * argument returned (the first on a tie), a clamp to [0, 1] has derivative 1
 * on [0, 1] and 0 outside.  The forward is the plain FP32 step, the adjoint
 * fields are FP64.
 *
 * vof_forward_record: nsteps steps from istep0 on the context's state (like
 * vof_run), storing a device checkpoint of the state every checkpoint_every
 * steps (0: ceil(sqrt(nsteps))).  Device memory: ceil(nsteps/every) + every
 * states of five fields (and the FP64 pressure in the convergent modes), plus
 * the engine's work fields (allocated once); with the intermediates kept
 * (vof_adjoint_storage), every - 1 segment states of five FP32 fields and
 * every x five FP32 intermediate fields instead of every segment states; in
 * the plain mode with an even jacobi_iters, when 1/32 of the device memory
 * stays free, as much again for a second kept segment (the record then runs
 * the last two segments as the reverse pass would replay them, and that pass
 * replays neither).  In VOF_MODE_MIXED / FP64 the
 * pressure is taken as the exact solution of the mean-free system (its
 * adjoint is the same solve on the pressure's adjoint, to prm.tol; the state
 * pressure, only a warm start, gets a zero adjoint).
 *
 * vof_backward: the reverse pass of the recorded run from the context's
 * current (final) state; *loss = L, grad_g = dL/d(gx, gy, gz).  Replays each
 * segment from its checkpoint; a reversed step takes its intermediates (u*,
 * v*, w*, F between the FCT sweeps) from that replay when they are kept, else
 * recomputes them from the step's start state.  VOF_E_STATE without a
 * recorded run.
 *
 * vof_adjoint_download: dL/d(field) of the initial state (field F, U, V, W or
 * P), FP64, reference layout, to host memory; valid after vof_backward.
 */
int vof_forward_record(vof_ctx* ctx, int istep0, int nsteps, int checkpoint_every);
int vof_backward(vof_ctx* ctx, const double* box, double* loss, double* grad_g);
int vof_adjoint_download(vof_ctx* ctx, int field, double* dst);
/* Kernel launches of one reversed step (segment replay and recompute
 * included; the convergent modes' multigrid solves not counted); VOF_E_STATE
 * before the first vof_forward_record. */
int vof_adjoint_kernels_per_step(const vof_ctx* ctx);

/* Where the reverse pass takes each step's intermediates from, for the next
 * vof_forward_record: VOF_ADJ_AUTO (the default) keeps them when the tape
 * with them leaves 1/32 of the device memory free, VOF_ADJ_RECOMPUTE always
 * recomputes them, VOF_ADJ_KEEP always keeps them (VOF_E_NOMEM from
 * vof_forward_record when they do not fit).  The gradients do not depend on
 * the choice.  vof_adjoint_keeps: 1 when the recorded tape keeps them, 0 when
 * it recomputes them, VOF_E_STATE before the first vof_forward_record. */
/* The FCT sweep adjoint has two kernels with the same results: a march along
 * each grid line (one thread per line; grids with at least 16384 lines per
 * sweep direction) and a shared-memory kernel (threads along lines; smaller
 * grids).  The environment variable VOF_ADJ_SWEEP=march or =shared, read when
 * a context's adjoint engine is created, forces one of them (a diagnostic
 * override). */
#define VOF_ADJ_AUTO      0
#define VOF_ADJ_RECOMPUTE 1
#define VOF_ADJ_KEEP      2
int vof_adjoint_storage(vof_ctx* ctx, int policy);
int vof_adjoint_keeps(const vof_ctx* ctx);

/* cudaError_t of the most recent failing CUDA call in this context (0 if none). */
int vof_last_cuda_error(const vof_ctx* ctx);

/* Fault injection for tests; no counterpart in the reference, whose set-up
 * (alloc_field, voftrial1.cu:1176-1203) exits on the first failing
 * cudaMalloc.  The context's own device allocations in the next vof_create
 * are numbered from 0; the one numbered n fails as if the device were out of
 * memory, and vof_create frees what it had allocated and returns
 * VOF_E_NOMEM.  The count includes the multigrid solver's allocations of
 * the convergent modes.  The next vof_create consumes the setting (one
 * atomic exchange) whether it fires or not; n < 0 clears it.  The setting is
 * process-wide: with several threads creating contexts, whichever create
 * comes first takes it. */
int vof_debug_fail_alloc(int n);

/* Failure-path check for tests; no counterpart in the reference, which has
 * no device-side waits.  Enqueues on the context's stream one kernel whose
 * only wait can never be satisfied: an mbarrier that expects asynchronous
 * copy bytes nothing will deliver, polled at most `limit` times (capped at
 * the library's own limit) by the same bounded wait the TMA kernels use.
 * When the wait runs out the kernel sets the context's device status word,
 * so the next vof_sync (or vof_reduce) returns VOF_E_TIMEOUT and clears it;
 * the context stays usable.  No copy is in flight at any time. */
int vof_debug_wait_timeout(vof_ctx* ctx, unsigned limit);

/* Number of kernel launches one vof_step enqueues for the current settings. */
int vof_kernels_per_step(const vof_ctx* ctx);

/* Device bytes held by the context. */
size_t vof_device_bytes(const vof_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* VOF_B200_H */
