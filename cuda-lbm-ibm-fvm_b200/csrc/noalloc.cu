// noalloc.cu -- one plain step without any allocation (vof_step_noalloc).
//
// Who needs this: callers that must not allocate device memory while they
// step -- a host program whose GPU memory is owned up front by its own pool
// or allocator, a tight control loop that cannot afford cudaMalloc's implicit
// device-wide synchronisation and latency, or code that has to stay clear of
// the driver allocator for any other reason.  They keep F, u, v, w and p in
// their own device buffers (reference layout) and call this entry point;
// everything else the step needs lives in g_arena below.
//
// The arena is a file-scope __device__ array of NOALLOC_ARENA_FLOATS floats
// (8 MiB), held by every GPU that loads the library until the process exits.
// In host code its name is only a host-side stand-in, so its device address
// is looked up with cudaGetSymbolAddress -- once per device, by the first
// call made on that device (with that device current).  That first call
// should come before any stream capture.  All calls share the arena and it
// keeps the last call's contents: each call clears the part it uses before
// using it, and calls that overlap on the GPU (two streams, two threads)
// race on it.  The call synchronises the given stream (it reads back the
// density table and the kernels' status word).
#include <cuda.h>
#include <cuda_runtime.h>
#include <string.h>

#include <mutex>

#include "../../include/vof.h"
#include "jacobi_tb.h"
#include "plain_step.h"
#include "tma.cuh"

namespace {

constexpr size_t NOALLOC_ARENA_FLOATS = VOF_NOALLOC_ARENA_FLOATS;  // 8 MiB
constexpr int NOALLOC_MAX_DEVICES = 64;
constexpr int NOALLOC_FIELDS = 11;  // F u v w u* v* w* rhs p0 p1 p2
constexpr int NOALLOC_TAIL = 64;    // density table (6 floats) + status word, 256-byte aligned

static __device__ __align__(256) float g_arena[NOALLOC_ARENA_FLOATS];

std::mutex g_mu;
float* g_base[NOALLOC_MAX_DEVICES] = {};

// Device address of g_arena on the current device (set up on first use).
int arena_base(float** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return VOF_E_CUDA;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return VOF_E_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_base[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_arena) != cudaSuccess) return VOF_E_CUDA;
        if (vof::plain_configure(0) != cudaSuccess) return VOF_E_CUDA;
        g_base[dev] = static_cast<float*>(p);
    }
    *out = g_base[dev];
    return VOF_OK;
}

int check_params(const vof_params* p) {
    if (!p) return VOF_E_INVALID;
    if (p->nx < 1 || p->ny < 1 || p->nz < 1) return VOF_E_SIZE;
    if (p->imin != 1 || p->jmin != 1 || p->kmin != 1 || p->imax != p->nx || p->jmax != p->ny || p->kmax != p->nz)
        return VOF_E_INVALID;
    if ((long long)p->nTot != (long long)(p->nx + 2) * (p->ny + 2) * (p->nz + 2)) return VOF_E_INVALID;
    if (!(p->dt > 0.0f) || !(p->dx > 0.0f) || !(p->dy > 0.0f) || !(p->dz > 0.0f)) return VOF_E_INVALID;
    if (p->jacobi_iters < 0 || p->jacobi_iters > 100000) return VOF_E_INVALID;
    if (p->mode != VOF_MODE_PLAIN) return VOF_E_UNSUPPORTED;
    if (p->surface_tension != 0) return VOF_E_UNSUPPORTED;  // its fields would need allocation
    return VOF_OK;
}

}  // namespace

extern "C" int vof_step_noalloc(const vof_params* prm, float* F, float* u, float* v, float* w, float* p,
                                int istep, void* stream) {
    int st = check_params(prm);
    if (st != VOF_OK) return st;
    if (!F || !u || !v || !w || !p) return VOF_E_INVALID;

    vof::Geom g;
    memset(&g, 0, sizeof(g));
    g.nx = prm->nx;
    g.ny = prm->ny;
    g.nz = prm->nz;
    g.px = (prm->nx + 2 + 31) / 32 * 32;
    g.py = prm->ny + 2;
    g.plane = g.px * g.py;
    g.dt = prm->dt;
    g.dx = prm->dx;
    g.dy = prm->dy;
    g.dz = prm->dz;
    g.dxi = prm->dxi;
    g.dyi = prm->dyi;
    g.dzi = prm->dzi;
    g.rho_l = prm->rho_l;
    g.rho_g = prm->rho_g;
    g.nu_l = prm->nu_l;
    g.nu_g = prm->nu_g;
    g.gx = prm->gx;
    g.gy = prm->gy;
    g.gz = prm->gz;
    // Size check: NOALLOC_FIELDS padded fields plus the tail must fit.
    const size_t elems = (size_t)g.plane * (size_t)(prm->nz + 2);
    if (elems > NOALLOC_ARENA_FLOATS / NOALLOC_FIELDS ||
        NOALLOC_FIELDS * elems + NOALLOC_TAIL > NOALLOC_ARENA_FLOATS || !vof::plain_supported(g))
        return VOF_E_SIZE;

    float* base = nullptr;
    if ((st = arena_base(&base)) != VOF_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float* f[NOALLOC_FIELDS];
    for (int q = 0; q < NOALLOC_FIELDS; ++q) f[q] = base + q * elems;
    float* tail = base + NOALLOC_FIELDS * elems;
    int* status = reinterpret_cast<int*>(tail + 8);

    // Clear everything this call uses: the previous call may have left
    // another grid's data, and the step relies on zero-filled scratch.
    cudaError_t e = cudaMemsetAsync(base, 0, (NOALLOC_FIELDS * elems + NOALLOC_TAIL) * sizeof(float), s);
    const size_t wref = (size_t)(prm->nx + 2) * sizeof(float), wpad = (size_t)g.px * sizeof(float);
    const size_t rows = (size_t)(prm->ny + 2) * (prm->nz + 2);
    float* user[5] = {F, u, v, w, p};
    const int slot_in[5] = {0, 1, 2, 3, 8};  // F u v w -> 0..3, p -> p0
    for (int q = 0; q < 5 && e == cudaSuccess; ++q)
        e = cudaMemcpy2DAsync(f[slot_in[q]], wpad, user[q], wref, wref, rows, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = vof::plain_density_pairs_on(&g, tail, s);
    if (e != cudaSuccess) return VOF_E_CUDA;

    CUtensorMap maps[4];
    const float* mapped[4] = {f[8], f[9], f[10], f[7]};
    for (int q = 0; q < 4; ++q)
        if (vof::jacobi_tb_maps(g, mapped[q], &maps[q]) != cudaSuccess) return VOF_E_UNSUPPORTED;

    vof::PlainBuffers b;
    memset(&b, 0, sizeof(b));
    b.F = f[0];
    b.u = f[1];
    b.v = f[2];
    b.w = f[3];
    b.us = f[4];
    b.vs = f[5];
    b.ws = f[6];
    b.rhs = f[7];
    b.p0 = f[8];
    b.p1 = f[9];
    b.p2 = f[10];
    b.maps = maps;
    b.status = status;
    int parity = 0;
    e = vof::plain_step(g, b, istep, prm->jacobi_iters, &parity, s, nullptr);
    // The status word first: on a timed-out wait the step's results are
    // invalid, and the caller's buffers keep the state they passed in.
    int dev_status = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&dev_status, status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return VOF_E_CUDA;
    if (dev_status) return VOF_E_TIMEOUT;
    float* pres = parity ? b.p1 : b.p0;
    float* out[5] = {b.F, b.u, b.v, b.w, pres};
    for (int q = 0; q < 5 && e == cudaSuccess; ++q)
        e = cudaMemcpy2DAsync(user[q], wref, out[q], wpad, wref, rows, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? VOF_OK : VOF_E_CUDA;
}
