// capi.cu -- the extern "C" boundary declared in include/vof.h.
//
// Owns the device buffers (the reference's DeviceFields, voftrial1.cu:1176-1226),
// converts between the reference layout and the padded internal layout, and
// sequences the step (voftrial1.cu:1361-1401) on the caller's stream, directly
// or through captured CUDA graphs.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <new>

#include "../../include/vof.h"
#include "jacobi_tb.h"
#include "adjoint.h"
#include "apply_bc.h"
#include "mg_solve.h"
#include "plain_step.h"
#include "reduce.h"
#include "tma.cuh"

using vof::Geom;

static_assert(sizeof(vof_params) == 144, "vof_params layout is part of the ABI");
static_assert(VOF_PHASES == vof::PLAIN_PHASES, "phase count");
static_assert(VOF_ADJ_AUTO == vof::ADJ_STORE_AUTO && VOF_ADJ_RECOMPUTE == vof::ADJ_STORE_RECOMPUTE &&
                  VOF_ADJ_KEEP == vof::ADJ_STORE_KEEP,
              "adjoint storage policy codes");

struct vof_ctx {
    vof_params prm;
    Geom g;
    int device;
    cudaStream_t stream;        // caller's stream (may be the legacy default stream)
    cudaStream_t cap_stream;    // private stream used only for graph capture
    vof::PlainBuffers b;
    int p_parity;               // which of p0/p1 holds the current pressure
    float* fields[VOF_NUM_FIELDS - 1];  // all but P (P depends on parity)
    float* stage;               // one field in the reference layout: host copies land here whole
    double* d_red_scratch;
    double* d_red_result;
    double* h_red_result;       // pinned, for vof_reduce
    int* d_status;              // device status word written by kernels (DEV_* codes)
    CUtensorMap maps[4];        // TMA descriptors: p0, p1, p2, rhs
    // convergent modes (VOF_MODE_MIXED / VOF_MODE_FP64)
    int conv;                   // nonzero in those modes
    double* p64;                // FP64 pressure (padded layout); p0 holds its FP32 copy
    vof::MgSolver mg;
    vof::MgStats stats;         // of the last pressure solve
    vof::AdjEngine* adj;        // adjoint engine (vof_forward_record / vof_backward), or null
    int adj_policy;             // VOF_ADJ_* for the next vof_forward_record
    cudaGraphExec_t graph[3][2];  // [istep % 3][p parity at step start]
    int last_cuda_error;
    size_t bytes;
    size_t elems;               // padded elements per field
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
        else prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int fail_cuda(vof_ctx* c, cudaError_t e) {
    if (c) c->last_cuda_error = (int)e;
    return VOF_E_CUDA;
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Largest interior extent accepted: keeps int32 indexing of the padded
// layout and the reference's int nTot (voftrial1.cu:40) from overflowing.
constexpr long long kMaxCells = 2000000000LL;

int validate(const vof_params* p) {
    if (!p) return VOF_E_INVALID;
    if (p->nx < 1 || p->ny < 1 || p->nz < 1) return VOF_E_SIZE;
    const long long pxl = round_up(p->nx + 2, 32);
    const long long tot = pxl * (p->ny + 2) * (long long)(p->nz + 2);
    if (tot > kMaxCells) return VOF_E_SIZE;
    if (p->imin != 1 || p->jmin != 1 || p->kmin != 1 || p->imax != p->nx || p->jmax != p->ny ||
        p->kmax != p->nz)
        return VOF_E_INVALID;
    if (p->nTot != (p->nx + 2) * (p->ny + 2) * (p->nz + 2)) return VOF_E_INVALID;
    if (!(p->dt > 0.0f) || !(p->dx > 0.0f) || !(p->dy > 0.0f) || !(p->dz > 0.0f)) return VOF_E_INVALID;
    if (p->jacobi_iters < 0 || p->jacobi_iters > 100000) return VOF_E_INVALID;
    if (p->mode != VOF_MODE_PLAIN && p->mode != VOF_MODE_MIXED && p->mode != VOF_MODE_FP64)
        return VOF_E_INVALID;
    if (p->mode != VOF_MODE_PLAIN && (!(p->tol > 0.0) || p->max_outer < 1 || p->max_outer > 100000))
        return VOF_E_INVALID;
    if (p->surface_tension != 0 && p->surface_tension != 1) return VOF_E_INVALID;
    return VOF_OK;
}

float* field_ptr(vof_ctx* c, int field) {
    if (field == VOF_FIELD_P) return c->p_parity ? c->b.p1 : c->b.p0;
    if (field < 0 || field >= VOF_NUM_FIELDS) return nullptr;
    const int slot = field < VOF_FIELD_P ? field : field - 1;
    return c->fields[slot];
}

void free_ctx(vof_ctx* c) {
    if (!c) return;
    for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 2; ++q)
            if (c->graph[r][q]) cudaGraphExecDestroy(c->graph[r][q]);
    for (int f = 0; f < VOF_NUM_FIELDS - 1; ++f)
        if (c->fields[f]) cudaFree(c->fields[f]);
    if (c->b.p0) cudaFree(c->b.p0);
    if (c->b.p1) cudaFree(c->b.p1);
    if (c->b.p2) cudaFree(c->b.p2);
    if (c->stage) cudaFree(c->stage);
    for (int q = 0; q < 4; ++q)
        if (c->b.csf[q]) cudaFree(c->b.csf[q]);
    if (c->d_red_scratch) cudaFree(c->d_red_scratch);
    if (c->d_red_result) cudaFree(c->d_red_result);
    if (c->h_red_result) cudaFreeHost(c->h_red_result);
    if (c->d_status) cudaFree(c->d_status);
    if (c->p64) cudaFree(c->p64);
    vof::mg_destroy(&c->mg);
    if (c->adj) {
        vof::adj_destroy(c->adj);
        delete c->adj;
    }
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    delete c;
}

// Layout conversion of one field on the device: `rows` rows of `width`
// floats from pitch spitch to pitch dpitch (reference layout <-> padded
// layout).  Host copies move the reference-layout field whole, in one
// contiguous cudaMemcpyAsync through the context's staging buffer, and this
// kernel repacks it: a row of (nx+2) floats is 808 bytes at 200^3, and
// row-by-row host copies of that size run far below the link's bandwidth.
__global__ void __launch_bounds__(256) k_repack(const float* __restrict__ src, int spitch, float* __restrict__ dst,
                                                int dpitch, int width, int rows) {
    for (int r = blockIdx.x * 8 + threadIdx.y; r < rows; r += gridDim.x * 8) {
        const float* a = src + (size_t)r * spitch;
        float* b = dst + (size_t)r * dpitch;
        for (int i = threadIdx.x; i < width; i += 32) b[i] = a[i];
    }
}

cudaError_t repack(const float* src, int spitch, float* dst, int dpitch, int width, int rows, cudaStream_t s) {
    int blocks = (rows + 7) / 8;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_repack<<<blocks, dim3(32, 8), 0, s>>>(src, spitch, dst, dpitch, width, rows);
    return cudaGetLastError();
}

// vof_debug_wait_timeout's kernel: one wait that can only run out.  The
// mbarrier expects 16 bytes of asynchronous copies that nothing issues, so
// after `limit` tries the wait gives up and the kernel records
// DEV_TMA_TIMEOUT in the context's status word, exactly as the blocked
// Jacobi kernel does when a TMA load does not land in time (mbar_wait of
// tma.cuh, the same bounded loop).  No copy is ever in flight.
__global__ void k_wait_unfed(int* status, uint32_t limit) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        vof::mbar_init(&bar, 1);
        vof::mbar_arrive_expect_tx(&bar, 16);
        if (!vof::mbar_wait(&bar, 0, limit)) atomicOr(status, vof::DEV_TMA_TIMEOUT);
    }
}

// Read (and clear) the device status word after the stream has drained.
int check_status(vof_ctx* c) {
    int st = 0;
    if (cudaMemcpy(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return VOF_E_CUDA;
    if (st == 0) return VOF_OK;
    cudaMemset(c->d_status, 0, sizeof(int));
    return VOF_E_TIMEOUT;
}

// One step of a convergent mode: predictor and rhs, the multigrid-accelerated
// FP64 defect correction for the pressure, correction and the FCT sweeps.
int conv_step(vof_ctx* c, int istep, cudaEvent_t* ev) {
    cudaError_t e = vof::plain_front(c->g, c->b, c->stream, ev);
    if (e != cudaSuccess) return fail_cuda(c, e);
    e = vof::mg_solve(c->g, c->mg, c->b.rhs, c->p64, c->b.p0, c->prm.tol, c->prm.max_outer, &c->stats, c->stream,
                       c->cap_stream);
    const bool not_conv = (e == cudaErrorNotReady);
    if (e != cudaSuccess && !not_conv) return fail_cuda(c, e);
    e = vof::plain_back(c->g, c->b, istep, c->b.p0, c->stream, ev);
    if (e != cudaSuccess) return fail_cuda(c, e);
    return not_conv ? VOF_E_NOT_CONVERGED : VOF_OK;
}

}  // namespace

extern "C" {

int vof_abi_version(void) { return VOF_ABI_VERSION; }

const char* vof_error_string(int status) {
    switch (status) {
        case VOF_OK: return "ok";
        case VOF_E_INVALID: return "invalid argument";
        case VOF_E_SIZE: return "grid size out of range";
        case VOF_E_NOMEM: return "out of memory";
        case VOF_E_CUDA: return "CUDA error (see vof_last_cuda_error)";
        case VOF_E_NOT_CONVERGED: return "iterative solve did not converge";
        case VOF_E_NONFINITE: return "non-finite value in the state";
        case VOF_E_STATE: return "call not valid in the current state";
        case VOF_E_UNSUPPORTED: return "unsupported mode or feature";
        case VOF_E_TIMEOUT: return "a device-side wait timed out (result invalid)";
        default: return "unknown status";
    }
}

int vof_params_finalize(vof_params* p) {
    if (!p) return VOF_E_INVALID;
    if (p->nx < 1 || p->ny < 1 || p->nz < 1) return VOF_E_SIZE;
    // voftrial1.cu:1262-1270, 1285-1291 (float expressions kept).
    p->imin = 1;
    p->imax = p->imin + p->nx - 1;
    p->jmin = 1;
    p->jmax = p->jmin + p->ny - 1;
    p->kmin = 1;
    p->kmax = p->kmin + p->nz - 1;
    p->dx = p->Lx / static_cast<float>(p->nx);
    p->dy = p->Ly / static_cast<float>(p->ny);
    p->dz = p->Lz / static_cast<float>(p->nz);
    p->dxi = 1.0f / p->dx;
    p->dyi = 1.0f / p->dy;
    p->dzi = 1.0f / p->dz;
    const long long tot = (long long)(p->nx + 2) * (p->ny + 2) * (p->nz + 2);
    if (tot > 0x7fffffffLL) return VOF_E_SIZE;
    p->nTot = (int)tot;
    return VOF_OK;
}

int vof_params_init(vof_params* p, int nx, int ny, int nz) {
    if (!p) return VOF_E_INVALID;
    memset(p, 0, sizeof(*p));
    p->nx = nx;
    p->ny = ny;
    p->nz = nz;
    // voftrial1.cu:1272-1283
    p->Lx = 0.1f;
    p->Ly = 0.1f;
    p->Lz = 0.1f;
    p->rho_l = 1000.0f;
    p->rho_g = 50.0f;
    p->nu_l = 1.0e-6f;
    p->nu_g = 1.5e-5f;
    p->sigma = 0.007f;
    p->gx = 0.0f;
    p->gy = -5.0f;
    p->gz = 0.0f;
    p->dt = 4.0e-6f;
    p->jacobi_iters = 10;  // voftrial1.cu:1371
    p->mode = VOF_MODE_PLAIN;
    p->inner_sweeps = 32;
    p->max_outer = 200;
    p->tol = 1e-8;
    p->surface_tension = 0;
    return vof_params_finalize(p);
}

// vof_debug_fail_alloc's setting: the number of the allocation of the next
// vof_create that fails (-1: none).
static std::atomic<int> g_fail_alloc_at{-1};

int vof_debug_fail_alloc(int n) {
    g_fail_alloc_at.store(n < 0 ? -1 : n);
    return VOF_OK;
}

int vof_create(const vof_params* p, void* stream, vof_ctx** out) {
    const int fail_at = g_fail_alloc_at.exchange(-1);  // consumed by this call
    if (!out) return VOF_E_INVALID;
    *out = nullptr;
    int st = validate(p);
    if (st != VOF_OK) return st;

    vof_ctx* c = new (std::nothrow) vof_ctx;
    if (!c) return VOF_E_NOMEM;
    memset(c, 0, sizeof(*c));
    c->prm = *p;
    c->stream = (cudaStream_t)stream;
    cudaError_t e = cudaGetDevice(&c->device);
    if (e != cudaSuccess) {
        free_ctx(c);
        return VOF_E_CUDA;
    }

    Geom& g = c->g;
    g.nx = p->nx;
    g.ny = p->ny;
    g.nz = p->nz;
    g.px = round_up(p->nx + 2, 32);
    g.py = p->ny + 2;
    g.plane = g.px * g.py;
    g.dt = p->dt;
    g.dx = p->dx;
    g.dy = p->dy;
    g.dz = p->dz;
    g.dxi = p->dxi;
    g.dyi = p->dyi;
    g.dzi = p->dzi;
    g.rho_l = p->rho_l;
    g.rho_g = p->rho_g;
    g.nu_l = p->nu_l;
    g.nu_g = p->nu_g;
    g.gx = p->gx;
    g.gy = p->gy;
    g.gz = p->gz;
    g.csf = p->surface_tension;
    g.sigma = p->sigma;
    if (!vof::plain_supported(g)) {
        free_ctx(c);
        return VOF_E_SIZE;
    }

    c->elems = (size_t)g.plane * (size_t)(p->nz + 2);
    const size_t fbytes = c->elems * sizeof(float);
    int alloc_no = 0;
    auto alloc = [&](void** ptr, size_t bytes) -> bool {
        if (alloc_no++ == fail_at) return false;  // injected (vof_debug_fail_alloc)
        if (cudaMalloc(ptr, bytes) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        c->bytes += bytes;
        return cudaMemsetAsync(*ptr, 0, bytes, c->stream) == cudaSuccess;
    };
    bool ok = true;
    for (int f = 0; f < VOF_NUM_FIELDS - 1 && ok; ++f) ok = alloc((void**)&c->fields[f], fbytes);
    ok = ok && alloc((void**)&c->b.p0, fbytes) && alloc((void**)&c->b.p1, fbytes) &&
         alloc((void**)&c->b.p2, fbytes);
    for (int q = 0; q < 4 && ok && g.csf; ++q) ok = alloc((void**)&c->b.csf[q], fbytes);
    ok = ok && alloc((void**)&c->stage, (size_t)p->nTot * sizeof(float));
    ok = ok && alloc((void**)&c->d_red_scratch, sizeof(double) * vof::RED_SCRATCH_DOUBLES);
    ok = ok && alloc((void**)&c->d_red_result, sizeof(double) * vof::RED_RESULT_DOUBLES);
    ok = ok && alloc((void**)&c->d_status, sizeof(int));
    c->conv = (p->mode != VOF_MODE_PLAIN);
    if (ok && c->conv) {
        ok = alloc((void**)&c->p64, c->elems * sizeof(double));
        if (ok && vof::mg_create(g, p->mode == VOF_MODE_MIXED ? vof::MG_MIXED : vof::MG_FP64, &c->mg, c->stream,
                                 &c->bytes, &alloc_no, fail_at) != cudaSuccess)
            ok = false;
    }
    if (ok && cudaMallocHost((void**)&c->h_red_result, sizeof(double) * 4) != cudaSuccess) ok = false;
    if (!ok) {
        free_ctx(c);
        return VOF_E_NOMEM;
    }
    c->b.F = c->fields[VOF_FIELD_F];
    c->b.u = c->fields[VOF_FIELD_U];
    c->b.v = c->fields[VOF_FIELD_V];
    c->b.w = c->fields[VOF_FIELD_W];
    c->b.us = c->fields[VOF_FIELD_USTAR - 1];
    c->b.vs = c->fields[VOF_FIELD_VSTAR - 1];
    c->b.ws = c->fields[VOF_FIELD_WSTAR - 1];
    c->b.rhs = c->fields[VOF_FIELD_RHS - 1];
    c->b.maps = c->maps;
    c->b.status = c->d_status;
    c->p_parity = 0;
    {
        const float* mapped[4] = {c->b.p0, c->b.p1, c->b.p2, c->b.rhs};
        for (int q = 0; q < 4; ++q) {
            if ((e = vof::jacobi_tb_maps(c->g, mapped[q], &c->maps[q])) != cudaSuccess) {
                c->last_cuda_error = (int)e;
                free_ctx(c);
                return VOF_E_UNSUPPORTED;
            }
        }
    }

    const int maxn = p->nx > p->ny ? (p->nx > p->nz ? p->nx : p->nz) : (p->ny > p->nz ? p->ny : p->nz);
    if ((e = vof::plain_configure(maxn)) != cudaSuccess || (e = vof::plain_density_pairs(&c->g)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
        c->last_cuda_error = (int)e;
        free_ctx(c);
        return VOF_E_CUDA;
    }
    *out = c;
    return VOF_OK;
}

void vof_destroy(vof_ctx* ctx) {
    if (!ctx) return;
    DeviceGuard dg(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    free_ctx(ctx);
}

int vof_get_params(const vof_ctx* ctx, vof_params* out) {
    if (!ctx || !out) return VOF_E_INVALID;
    *out = ctx->prm;
    return VOF_OK;
}

int vof_upload(vof_ctx* ctx, int field, const float* src, int src_is_device) {
    if (!ctx || !src) return VOF_E_INVALID;
    float* dst = field_ptr(ctx, field);
    if (!dst) return VOF_E_INVALID;
    DeviceGuard dg(ctx->device);
    const Geom& g = ctx->g;
    const int rows = (g.ny + 2) * (g.nz + 2);
    cudaError_t e = cudaSuccess;
    const float* from = src;
    if (!src_is_device) {  // one contiguous copy of the whole field, then the repack
        e = cudaMemcpyAsync(ctx->stage, src, (size_t)ctx->prm.nTot * sizeof(float), cudaMemcpyHostToDevice,
                            ctx->stream);
        from = ctx->stage;
    }
    if (e == cudaSuccess) e = repack(from, g.nx + 2, dst, g.px, g.nx + 2, rows, ctx->stream);
    if (e == cudaSuccess && ctx->conv && field == VOF_FIELD_P) e = vof::mg_widen(g, ctx->mg, dst, ctx->p64, ctx->stream);
    return e == cudaSuccess ? VOF_OK : fail_cuda(ctx, e);
}

int vof_download(vof_ctx* ctx, int field, float* dst, int dst_is_device) {
    if (!ctx || !dst) return VOF_E_INVALID;
    float* src = field_ptr(ctx, field);
    if (!src) return VOF_E_INVALID;
    DeviceGuard dg(ctx->device);
    const Geom& g = ctx->g;
    const int rows = (g.ny + 2) * (g.nz + 2);
    cudaError_t e = repack(src, g.px, dst_is_device ? dst : ctx->stage, g.nx + 2, g.nx + 2, rows, ctx->stream);
    if (e == cudaSuccess && !dst_is_device) {  // the repacked field in one contiguous copy
        e = cudaMemcpyAsync(dst, ctx->stage, (size_t)ctx->prm.nTot * sizeof(float), cudaMemcpyDeviceToHost,
                            ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    return e == cudaSuccess ? VOF_OK : fail_cuda(ctx, e);
}

int vof_get_planes(vof_ctx* ctx, int field, int k0, int nk, float* dst, int dst_is_device) {
    if (!ctx || !dst || nk < 1 || k0 < 0 || k0 + nk > ctx->g.nz + 2) return VOF_E_INVALID;
    const float* src = field_ptr(ctx, field);
    if (!src) return VOF_E_INVALID;
    DeviceGuard dg(ctx->device);
    const Geom& g = ctx->g;
    const int rows = (g.ny + 2) * nk;
    cudaError_t e = repack(src + (size_t)k0 * g.plane, g.px, dst_is_device ? dst : ctx->stage, g.nx + 2, g.nx + 2,
                           rows, ctx->stream);
    if (e == cudaSuccess && !dst_is_device) {
        e = cudaMemcpyAsync(dst, ctx->stage, (size_t)rows * (g.nx + 2) * sizeof(float), cudaMemcpyDeviceToHost,
                            ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    return e == cudaSuccess ? VOF_OK : fail_cuda(ctx, e);
}

int vof_put_planes(vof_ctx* ctx, int field, int k0, int nk, const float* src, int src_is_device) {
    if (!ctx || !src || nk < 1 || k0 < 0 || k0 + nk > ctx->g.nz + 2) return VOF_E_INVALID;
    float* dst = field_ptr(ctx, field);
    if (!dst) return VOF_E_INVALID;
    if (ctx->conv && field == VOF_FIELD_P) return VOF_E_UNSUPPORTED;  // its FP64 copy is the state there
    DeviceGuard dg(ctx->device);
    const Geom& g = ctx->g;
    const int rows = (g.ny + 2) * nk;
    cudaError_t e = cudaSuccess;
    const float* from = src;
    if (!src_is_device) {
        e = cudaMemcpyAsync(ctx->stage, src, (size_t)rows * (g.nx + 2) * sizeof(float), cudaMemcpyHostToDevice,
                            ctx->stream);
        from = ctx->stage;
    }
    if (e == cudaSuccess) e = repack(from, g.nx + 2, dst + (size_t)k0 * g.plane, g.px, g.nx + 2, rows, ctx->stream);
    return e == cudaSuccess ? VOF_OK : fail_cuda(ctx, e);
}

int vof_step(vof_ctx* ctx, int istep) {
    if (!ctx) return VOF_E_INVALID;
    DeviceGuard dg(ctx->device);
    if (ctx->conv) return conv_step(ctx, istep, nullptr);
    cudaError_t e = vof::plain_step(ctx->g, ctx->b, istep, ctx->prm.jacobi_iters, &ctx->p_parity,
                                    ctx->stream);
    return e == cudaSuccess ? VOF_OK : fail_cuda(ctx, e);
}

int vof_run(vof_ctx* ctx, int istep0, int nsteps) {
    if (!ctx || nsteps < 0) return VOF_E_INVALID;
    DeviceGuard dg(ctx->device);
    if (ctx->conv) {  // data-dependent solver loop: plain launches, no graphs
        for (int s = 0; s < nsteps; ++s) {
            const int st = conv_step(ctx, istep0 + s, nullptr);
            if (st != VOF_OK) return st;
        }
        return VOF_OK;
    }
    for (int s = 0; s < nsteps; ++s) {
        const int istep = istep0 + s;
        const int r = ((istep % 3) + 3) % 3;
        const int par = ctx->p_parity;
        if (!ctx->graph[r][par]) {
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return fail_cuda(ctx, e);
            int tmp_parity = par;
            cudaError_t le = vof::plain_step(ctx->g, ctx->b, istep, ctx->prm.jacobi_iters, &tmp_parity,
                                             ctx->cap_stream);
            e = cudaStreamEndCapture(ctx->cap_stream, &graph);
            if (le != cudaSuccess) e = le;
            if (e != cudaSuccess) {
                if (graph) cudaGraphDestroy(graph);
                return fail_cuda(ctx, e);
            }
            e = cudaGraphInstantiate(&ctx->graph[r][par], graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) {
                ctx->graph[r][par] = nullptr;
                return fail_cuda(ctx, e);
            }
        }
        cudaError_t e = cudaGraphLaunch(ctx->graph[r][par], ctx->stream);
        if (e != cudaSuccess) return fail_cuda(ctx, e);
        ctx->p_parity = par ^ (ctx->prm.jacobi_iters & 1);
    }
    return VOF_OK;
}

int vof_step_timed(vof_ctx* ctx, int istep, float* phase_ms, int* launches, int nphase) {
    if (!ctx || nphase < 0) return VOF_E_INVALID;
    DeviceGuard dg(ctx->device);
    cudaEvent_t ev[vof::PLAIN_PHASES + 1] = {};
    cudaError_t e = cudaSuccess;
    for (int q = 0; q <= vof::PLAIN_PHASES && e == cudaSuccess; ++q) e = cudaEventCreate(&ev[q]);
    int conv_status = VOF_OK;
    if (e == cudaSuccess && ctx->conv) {
        conv_status = conv_step(ctx, istep, ev);
        if (conv_status == VOF_E_CUDA) e = (cudaError_t)ctx->last_cuda_error;
    } else if (e == cudaSuccess) {
        e = vof::plain_step(ctx->g, ctx->b, istep, ctx->prm.jacobi_iters, &ctx->p_parity, ctx->stream, ev);
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(ev[vof::PLAIN_PHASES]);
    const int n = nphase < VOF_PHASES ? nphase : VOF_PHASES;
    for (int q = 0; q < n && e == cudaSuccess; ++q) {
        float ms = 0.0f;
        e = cudaEventElapsedTime(&ms, ev[q], ev[q + 1]);
        if (phase_ms) phase_ms[q] = ms;
        if (launches)
            launches[q] = (ctx->conv && q == vof::PHASE_JACOBI)
                              ? ctx->stats.launches
                              : vof::plain_phase_launches(ctx->g, q, ctx->prm.jacobi_iters);
    }
    for (int q = 0; q <= vof::PLAIN_PHASES; ++q)
        if (ev[q]) cudaEventDestroy(ev[q]);
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    if (conv_status != VOF_OK) return conv_status;
    return n;
}

const char* vof_phase_name(int phase) {
    static const char* names[VOF_PHASES] = {"predict", "rhs", "jacobi", "correct", "sweep1", "sweep2", "sweep3"};
    return (phase >= 0 && phase < VOF_PHASES) ? names[phase] : nullptr;
}

int vof_sync(vof_ctx* ctx) {
    if (!ctx) return VOF_E_INVALID;
    DeviceGuard dg(ctx->device);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    return check_status(ctx);
}

// The reduction `what` over the interior cells of planes k0..k1 (1..nz: the
// whole grid), stream-ordered, its value written to *host_out when the stream
// gets there.  Page-locked host memory mapped into the device is written by
// the reduction kernel itself; any other address gets a copy in the stream.
static int reduce_planes_async(vof_ctx* ctx, int what, int k0, int k1, double* host_out) {
    DeviceGuard dg(ctx->device);
    // the planes k0..k1 as a grid of their own: the same rows, the base moved
    // k0 - 1 planes up (every reduction here reads a cell and its upper faces)
    Geom sub = ctx->g;
    sub.nz = k1 - k0 + 1;
    const size_t off = (size_t)(k0 - 1) * ctx->g.plane;
    vof::ReduceInputs in;
    in.F = ctx->b.F + off;
    in.u = ctx->b.u + off;
    in.v = ctx->b.v + off;
    in.w = ctx->b.w + off;
    in.p = (ctx->p_parity ? ctx->b.p1 : ctx->b.p0) + off;
    in.rhs = ctx->b.rhs + off;
    double* alias = nullptr;
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, host_out) == cudaSuccess) {
        if (pa.type == cudaMemoryTypeHost && pa.devicePointer) alias = static_cast<double*>(pa.devicePointer);
    } else {
        cudaGetLastError();  // not a pointer CUDA knows: an ordinary host address
    }
    bool wrote = false;
    cudaError_t e = vof::reduce_launch(sub, in, what, ctx->d_red_scratch, ctx->d_red_result, ctx->stream, alias,
                                       &wrote);
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    if (wrote) return VOF_OK;
    e = cudaMemcpyAsync(host_out, ctx->d_red_result + vof::reduce_result_slot(what), sizeof(double),
                        cudaMemcpyDeviceToHost, ctx->stream);
    return e == cudaSuccess ? VOF_OK : fail_cuda(ctx, e);
}

// The reductions a plane range supports: those whose every term is one cell
// and the faces above it.
static int check_range(const vof_ctx* ctx, int what, int k0, int k1) {
    if (k0 < 1 || k1 > ctx->g.nz || k0 > k1) return VOF_E_INVALID;
    if (what != VOF_RED_VOLUME && what != VOF_RED_F_MIN && what != VOF_RED_F_MAX && what != VOF_RED_DIV_L2 &&
        what != VOF_RED_DIV_MAX)
        return what >= 0 && what < VOF_NUM_REDUCTIONS ? VOF_E_UNSUPPORTED : VOF_E_INVALID;
    return VOF_OK;
}

int vof_reduce_async(vof_ctx* ctx, int what, double* host_out) {
    if (!ctx || !host_out) return VOF_E_INVALID;
    if (what < 0 || what >= VOF_NUM_REDUCTIONS) return VOF_E_INVALID;
    return reduce_planes_async(ctx, what, 1, ctx->g.nz, host_out);
}

int vof_reduce(vof_ctx* ctx, int what, double* out) {
    if (!ctx || !out) return VOF_E_INVALID;
    int st = vof_reduce_async(ctx, what, ctx->h_red_result);
    if (st != VOF_OK) return st;
    st = vof_sync(ctx);
    if (st != VOF_OK) return st;
    *out = ctx->h_red_result[0];
    return VOF_OK;
}

int vof_reduce_range_async(vof_ctx* ctx, int what, int k0, int k1, double* host_out) {
    if (!ctx || !host_out) return VOF_E_INVALID;
    const int st = check_range(ctx, what, k0, k1);
    if (st != VOF_OK) return st;
    return reduce_planes_async(ctx, what, k0, k1, host_out);
}

int vof_reduce_range(vof_ctx* ctx, int what, int k0, int k1, double* out) {
    if (!ctx || !out) return VOF_E_INVALID;
    int st = vof_reduce_range_async(ctx, what, k0, k1, ctx->h_red_result);
    if (st != VOF_OK) return st;
    st = vof_sync(ctx);
    if (st != VOF_OK) return st;
    *out = ctx->h_red_result[0];
    return VOF_OK;
}

int vof_apply_bc(vof_ctx* ctx) {
    if (!ctx) return VOF_E_INVALID;
    if (ctx->conv) return VOF_E_UNSUPPORTED;  // the pressure state is its FP64 copy there
    DeviceGuard dg(ctx->device);
    vof::BcFields f;
    f.u = field_ptr(ctx, VOF_FIELD_U);
    f.v = field_ptr(ctx, VOF_FIELD_V);
    f.w = field_ptr(ctx, VOF_FIELD_W);
    f.F = field_ptr(ctx, VOF_FIELD_F);
    f.p = field_ptr(ctx, VOF_FIELD_P);
    f.rho = nullptr;  // never stored: every kernel forms rho from F
    const cudaError_t e = vof::apply_bc_launch(ctx->g.nx, ctx->g.ny, ctx->g.nz, ctx->g.px, f, ctx->stream);
    return e == cudaSuccess ? VOF_OK : fail_cuda(ctx, e);
}

int vof_apply_bc_fields(const vof_params* p, float* u, float* v, float* w, float* F, float* pres, float* rho,
                        void* stream) {
    if (!p) return VOF_E_INVALID;
    if (p->nx < 1 || p->ny < 1 || p->nz < 1) return VOF_E_SIZE;
    if ((long long)(p->nx + 2) * (p->ny + 2) * (long long)(p->nz + 2) > kMaxCells) return VOF_E_SIZE;
    if (p->imin != 1 || p->jmin != 1 || p->kmin != 1 || p->imax != p->nx || p->jmax != p->ny || p->kmax != p->nz)
        return VOF_E_INVALID;
    if ((long long)p->nTot != (long long)(p->nx + 2) * (p->ny + 2) * (p->nz + 2)) return VOF_E_INVALID;
    const vof::BcFields f{u, v, w, F, pres, rho};
    const cudaError_t e =
        vof::apply_bc_launch(p->nx, p->ny, p->nz, p->nx + 2, f, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? VOF_OK : VOF_E_CUDA;
}

int vof_solver_stats(const vof_ctx* ctx, int* outer, double* rel_initial, double* rel_final) {
    if (!ctx) return VOF_E_INVALID;
    if (!ctx->conv) return VOF_E_STATE;
    if (outer) *outer = ctx->stats.outer;
    if (rel_initial) *rel_initial = ctx->stats.rel_initial;
    if (rel_final) *rel_final = ctx->stats.rel_final;
    return VOF_OK;
}

int vof_forward_record(vof_ctx* ctx, int istep0, int nsteps, int checkpoint_every) {
    if (!ctx || nsteps < 1 || checkpoint_every < 0) return VOF_E_INVALID;
    if (ctx->prm.surface_tension) return VOF_E_UNSUPPORTED;  // the adjoint has no surface-tension term
    DeviceGuard dg(ctx->device);
    cudaError_t e;
    if (!ctx->adj) {
        ctx->adj = new (std::nothrow) vof::AdjEngine();
        if (!ctx->adj) return VOF_E_NOMEM;
        e = vof::adj_create(ctx->g, ctx->prm.jacobi_iters, ctx->conv ? ctx->mg.mode : 0, ctx->prm.tol,
                            ctx->prm.max_outer, ctx->adj, ctx->stream);
        if (e != cudaSuccess) {
            vof::adj_destroy(ctx->adj);
            delete ctx->adj;
            ctx->adj = nullptr;
            return e == cudaErrorMemoryAllocation ? VOF_E_NOMEM : fail_cuda(ctx, e);
        }
    }
    vof::AdjEngine* A = ctx->adj;
    A->policy = ctx->adj_policy;
    if ((e = vof::adj_tape(A, istep0, nsteps, checkpoint_every, ctx->stream)) != cudaSuccess)
        return e == cudaErrorMemoryAllocation ? VOF_E_NOMEM : fail_cuda(ctx, e);
    int not_conv = 0;
    int m = 0;  // next checkpoint
    for (int n = 0; n < nsteps; ++n) {
        if (m < A->ncp && n == vof::adj_segment_first(*A, m)) {
            vof::AdjState x;
            for (int q = 0; q < 5; ++q) x.f[q] = field_ptr(ctx, q);
            x.p64 = ctx->conv ? ctx->p64 : nullptr;
            if ((e = vof::adj_save(A, m, x, ctx->stream)) != cudaSuccess) return fail_cuda(ctx, e);
            if (m == A->ncp - 1 && vof::adj_can_record_tail(*A)) {
                // the last segment runs as the reverse pass would replay it,
                // so that pass starts on it without a replay
                float* const extra[4] = {ctx->b.us, ctx->b.vs, ctx->b.ws, ctx->b.rhs};
                if ((e = vof::adj_record_tail(A, x, extra, ctx->stream)) != cudaSuccess) return fail_cuda(ctx, e);
                break;
            }
            if (vof::adj_can_keep(*A, m)) {
                // so do the segments before it that have a set of kept
                // buffers; the next pass of the loop is at the next
                // segment's first step
                if ((e = vof::adj_record_keep(A, m, x, ctx->stream)) != cudaSuccess) return fail_cuda(ctx, e);
                ++m;
                n = vof::adj_segment_first(*A, m) - 1;
                continue;
            }
            ++m;
        }
        if (ctx->conv) {
            const int st = conv_step(ctx, istep0 + n, nullptr);
            if (st == VOF_E_NOT_CONVERGED) not_conv = 1;
            else if (st != VOF_OK) return st;
        } else {
            e = vof::plain_step(ctx->g, ctx->b, istep0 + n, ctx->prm.jacobi_iters, &ctx->p_parity, ctx->stream);
            if (e != cudaSuccess) return fail_cuda(ctx, e);
        }
    }
    const int st = vof_sync(ctx);
    if (st != VOF_OK) return st;
    A->recorded = true;
    return not_conv ? VOF_E_NOT_CONVERGED : VOF_OK;
}

int vof_backward(vof_ctx* ctx, const double* box, double* loss, double* grad_g) {
    if (!ctx || !box) return VOF_E_INVALID;
    if (!ctx->adj || !ctx->adj->recorded) return VOF_E_STATE;
    DeviceGuard dg(ctx->device);
    vof::AdjState fin;
    for (int q = 0; q < 5; ++q) fin.f[q] = field_ptr(ctx, q);
    fin.p64 = ctx->conv ? ctx->p64 : nullptr;
    cudaError_t e = vof::adj_backward(ctx->adj, fin, box, loss, grad_g, ctx->stream);
    if (e == cudaErrorNotReady) return VOF_E_NOT_CONVERGED;
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    int st = 0;
    if (cudaMemcpy(&st, ctx->adj->status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return VOF_E_CUDA;
    if (st != 0) {
        cudaMemset(ctx->adj->status, 0, sizeof(int));
        return VOF_E_TIMEOUT;
    }
    return VOF_OK;
}

int vof_adjoint_download(vof_ctx* ctx, int field, double* dst) {
    if (!ctx || !dst || field < VOF_FIELD_F || field > VOF_FIELD_P) return VOF_E_INVALID;
    if (!ctx->adj || !ctx->adj->recorded) return VOF_E_STATE;
    DeviceGuard dg(ctx->device);
    const vof::AdjEngine* A = ctx->adj;
    const double* src[5] = {A->lF, A->lu, A->lv, A->lw, A->lp[A->lp_cur]};
    const Geom& g = ctx->g;
    const size_t w = (size_t)(g.nx + 2) * sizeof(double);
    cudaError_t e = cudaMemcpy2DAsync(dst, w, src[field], (size_t)g.px * sizeof(double), w,
                                      (size_t)(g.ny + 2) * (g.nz + 2), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? VOF_OK : fail_cuda(ctx, e);
}

int vof_adjoint_kernels_per_step(const vof_ctx* ctx) {
    if (!ctx) return VOF_E_INVALID;
    if (!ctx->adj) return VOF_E_STATE;
    return vof::adj_kernels_per_step(*ctx->adj);
}

int vof_adjoint_storage(vof_ctx* ctx, int policy) {
    if (!ctx || policy < VOF_ADJ_AUTO || policy > VOF_ADJ_KEEP) return VOF_E_INVALID;
    ctx->adj_policy = policy;
    return VOF_OK;
}

int vof_adjoint_keeps(const vof_ctx* ctx) {
    if (!ctx) return VOF_E_INVALID;
    if (!ctx->adj || !ctx->adj->cp) return VOF_E_STATE;
    return ctx->adj->keep ? 1 : 0;
}

int vof_debug_wait_timeout(vof_ctx* ctx, unsigned limit) {
    if (!ctx) return VOF_E_INVALID;
    DeviceGuard dg(ctx->device);
    k_wait_unfed<<<1, 32, 0, ctx->stream>>>(ctx->d_status, limit < vof::MBAR_SPIN_LIMIT ? limit : vof::MBAR_SPIN_LIMIT);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VOF_OK : fail_cuda(ctx, e);
}

int vof_last_cuda_error(const vof_ctx* ctx) { return ctx ? ctx->last_cuda_error : 0; }

int vof_kernels_per_step(const vof_ctx* ctx) {
    if (!ctx) return VOF_E_INVALID;
    if (ctx->conv) return 2 + ctx->stats.launches + 4;  // the last step's count
    return vof::plain_kernels_per_step(ctx->g, ctx->prm.jacobi_iters);
}

size_t vof_device_bytes(const vof_ctx* ctx) {
    return ctx ? ctx->bytes + (ctx->adj ? ctx->adj->bytes + ctx->adj->tape_bytes : 0) : 0;
}

}  // extern "C"
