// reduce.cu -- FP64 diagnostics over the step state (no reference counterpart:
// voftrial1.cu computes no reductions; the volume, divergence and residual
// monitors are additions of this library).
//
// Every reduction is deterministic: pass 1 runs a fixed grid of RED_BLOCKS
// blocks over a fixed cell->thread mapping, each block reducing with warp
// shuffles into one FP64 partial; pass 2 is one block that folds the partials
// in a fixed order.  The same inputs give the same bits on every run.
#include "reduce.h"

#include <cuda_runtime.h>
#include <math.h>

namespace vof {

constexpr int RED_THREADS = 256;

enum Op { OP_SUM = 0, OP_MAX = 1, OP_MIN = 2 };

__device__ __forceinline__ double combine(double a, double b, int op) {
    return op == OP_SUM ? a + b : (op == OP_MAX ? fmax(a, b) : fmin(a, b));
}

__device__ __forceinline__ double identity(int op) {
    return op == OP_SUM ? 0.0 : (op == OP_MAX ? -INFINITY : INFINITY);
}

// Block reduction of NV values per thread into partial[NV*blockIdx.x + v].
template <int NV>
__device__ void block_reduce_store(double (&val)[NV], const int (&op)[NV], double* partial) {
    __shared__ double sh[NV][RED_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        double x = val[v];
        for (int o = 16; o > 0; o >>= 1) x = combine(x, __shfl_down_sync(0xffffffffu, x, o), op[v]);
        if (lane == 0) sh[v][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double x = sh[v][0];
            for (int q = 1; q < RED_THREADS / 32; ++q) x = combine(x, sh[v][q], op[v]);
            partial[(size_t)NV * blockIdx.x + v] = x;
        }
    }
}

// Interior-cell iterator: the rows (j, k) are dealt to the warps of the grid
// in a fixed order (row r = (k-1) ny + j-1 to warp r mod the warp count), the
// lanes of a warp striding along x (unrolled by 4, so that several loads of a
// lane are in flight): coalesced loads and one integer division per row.  A
// fixed mapping for the fixed grid, so the sums are reproducible.
#define FOR_INTERIOR(g, i, j, k)                                                                        \
    for (int r_ = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nr_ = (g).ny * (g).nz,          \
             sr_ = (int)((gridDim.x * blockDim.x) >> 5);                                                \
         r_ < nr_; r_ += sr_)                                                                           \
        _Pragma("unroll 4") for (int j = 1 + r_ % (g).ny, k = 1 + r_ / (g).ny, i = 1 + (int)(threadIdx.x & 31); \
                                 i <= (g).nx; i += 32)

__global__ void __launch_bounds__(RED_THREADS) k_red_field(Geom g, const float* __restrict__ a,
                                                           double* partial) {
    // v0 = sum, v1 = max, v2 = min over interior cells.
    double val[3] = {0.0, -INFINITY, INFINITY};
    const int op[3] = {OP_SUM, OP_MAX, OP_MIN};
    FOR_INTERIOR(g, i, j, k) {
        const double x = (double)a[gidx(g, i, j, k)];
        val[0] += x;
        val[1] = fmax(val[1], x);
        val[2] = fmin(val[2], x);
    }
    block_reduce_store<3>(val, op, partial);
}

__global__ void __launch_bounds__(RED_THREADS) k_red_div(Geom g, const float* __restrict__ u,
                                                         const float* __restrict__ v,
                                                         const float* __restrict__ w,
                                                         double* partial) {
    double val[2] = {0.0, 0.0};
    const int op[2] = {OP_SUM, OP_MAX};
    const double dxi = g.dxi, dyi = g.dyi, dzi = g.dzi;
    FOR_INTERIOR(g, i, j, k) {
        const int id = gidx(g, i, j, k);
        const double d = ((double)u[id + 1] - (double)u[id]) * dxi +
                         ((double)v[id + g.px] - (double)v[id]) * dyi +
                         ((double)w[id + g.plane] - (double)w[id]) * dzi;
        val[0] += d * d;
        val[1] = fmax(val[1], fabs(d));
    }
    block_reduce_store<2>(val, op, partial);
}

// Residual of the pressure system A p = b, b = rhs - mean(rhs), with A the
// Neumann operator of the Jacobi sweep (voftrial1.cu:424-430):
// (A p)_c = sum over non-wall neighbours nb of a_nb (p_nb - p_c).
__global__ void __launch_bounds__(RED_THREADS) k_red_resid(Geom g, const float* __restrict__ rhs,
                                                           const float* __restrict__ p,
                                                           const double* __restrict__ mean,
                                                           double* partial) {
    double val[2] = {0.0, 0.0};
    const int op[2] = {OP_SUM, OP_SUM};
    const double m = *mean;
    const double cx = (double)g.dxi * g.dxi, cy = (double)g.dyi * g.dyi, cz = (double)g.dzi * g.dzi;
    FOR_INTERIOR(g, i, j, k) {
        const int id = gidx(g, i, j, k);
        const double pc = p[id];
        double ap = 0.0;
        if (i != g.nx) ap += cx * ((double)p[id + 1] - pc);
        if (i != 1) ap += cx * ((double)p[id - 1] - pc);
        if (j != g.ny) ap += cy * ((double)p[id + g.px] - pc);
        if (j != 1) ap += cy * ((double)p[id - g.px] - pc);
        if (k != g.nz) ap += cz * ((double)p[id + g.plane] - pc);
        if (k != 1) ap += cz * ((double)p[id - g.plane] - pc);
        const double b = (double)rhs[id] - m;
        const double r = b - ap;
        val[0] += r * r;
        val[1] += b * b;
    }
    block_reduce_store<2>(val, op, partial);
}

__global__ void __launch_bounds__(RED_THREADS) k_red_nonfinite(Geom g, const float* __restrict__ f0,
                                                               const float* __restrict__ f1,
                                                               const float* __restrict__ f2,
                                                               const float* __restrict__ f3,
                                                               const float* __restrict__ f4,
                                                               double* partial) {
    double val[1] = {0.0};
    const int op[1] = {OP_SUM};
    // every cell with its ghosts: rows (j, k) of ny+2 x nz+2 to the warps, lanes along x
    const int nrow = (g.ny + 2) * (g.nz + 2), srow = (int)((gridDim.x * blockDim.x) >> 5);
    for (int r = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); r < nrow; r += srow) {
        const int row = gidx(g, 0, r % (g.ny + 2), r / (g.ny + 2));
        for (int i = (int)(threadIdx.x & 31); i <= g.nx + 1; i += 32) {
            const int id = row + i;
            val[0] += (double)(!isfinite(f0[id])) + (double)(!isfinite(f1[id])) +
                      (double)(!isfinite(f2[id])) + (double)(!isfinite(f3[id])) +
                      (double)(!isfinite(f4[id]));
        }
    }
    block_reduce_store<1>(val, op, partial);
}

// Pass 2: fold nblk partials of NV values; result[v] for each v.  Optional
// post-processing: MODE_MEAN divides result[0] by count, MODE_SQRT takes the
// square root of result[0], MODE_RATIO = sqrt(result[0] / result[1]),
// MODE_VOLUME multiplies result[0] by the cell volume.
enum Post { POST_NONE = 0, POST_MEAN = 1, POST_SQRT = 2, POST_RATIO = 3, POST_SCALE = 4 };

// The fold of pass 2 by one block of RED_THREADS threads (partials read past
// L1: they may have been written by other blocks of the same launch).
// Each thread folds its strided partials in order, the warps fold their
// lanes by a fixed shuffle tree, and thread 0 folds the warps in order.
__device__ void fold_partials(const double* __restrict__ partial, int nblk, int nv, int op0, int op1, int op2,
                              int post, double scale, double* result) {
    __shared__ double sh[3][RED_THREADS / 32];
    const int ops[3] = {op0, op1, op2};
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // the partials of a thread loaded together, then folded in order
    constexpr int PER = (RED_BLOCKS + RED_THREADS - 1) / RED_THREADS;
    double xs[3][PER];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int b = threadIdx.x + q * RED_THREADS;
            xs[v][q] = (v < nv && b < nblk) ? __ldcg(partial + (size_t)nv * b + v) : identity(ops[v]);
        }
    for (int v = 0; v < nv; ++v) {
        double x = identity(ops[v]);
#pragma unroll
        for (int q = 0; q < PER; ++q) x = combine(x, xs[v][q], ops[v]);
        for (int b = threadIdx.x + PER * RED_THREADS; b < nblk; b += RED_THREADS)
            x = combine(x, __ldcg(partial + (size_t)nv * b + v), ops[v]);
        for (int o = 16; o > 0; o >>= 1) x = combine(x, __shfl_down_sync(0xffffffffu, x, o), ops[v]);
        if (lane == 0) sh[v][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r[3];
        for (int v = 0; v < nv; ++v) {
            double x = sh[v][0];
            for (int q = 1; q < RED_THREADS / 32; ++q) x = combine(x, sh[v][q], ops[v]);
            r[v] = x;
        }
        double out0 = r[0];
        if (post == POST_MEAN) out0 = r[0] * scale;
        else if (post == POST_SQRT) out0 = sqrt(r[0]);
        else if (post == POST_RATIO) out0 = (r[1] > 0.0) ? sqrt(r[0] / r[1]) : 0.0;
        else if (post == POST_SCALE) out0 = r[0] * scale;
        result[0] = out0;
        for (int v = 1; v < nv; ++v) result[v] = r[v];
    }
}

__global__ void __launch_bounds__(RED_THREADS) k_red_finish(const double* __restrict__ partial,
                                                            int nblk, int nv, int op0, int op1,
                                                            int op2, int post, double scale,
                                                            double* result) {
    fold_partials(partial, nblk, nv, op0, op1, op2, post, scale, result);
}

// k_red_field and k_red_finish in one launch: every block stores its partial
// and counts itself done; the last one folds all partials in the same fixed
// order as k_red_finish (the same bits), copies result[slot] to the mapped
// host double when given, and clears the counter for the next launch.
// The field is read as aligned float4 words (a padded row starts on a
// 128-byte boundary and holds at least round_up(nx + 2, 4) floats): rows
// dealt to warps as in FOR_INTERIOR, the lanes on consecutive words of a row,
// the ghost and padding entries masked out.  A warp loads RG rows x 2 words
// per lane before it adds any of them, so that 4 loads of a lane are in
// flight at once (more spill at 64 registers, the cap for 4 blocks per SM);
// a row wider than 64 words takes several such passes.
constexpr int RG = 2;

__device__ __forceinline__ void field_words(const Geom& g, const float* __restrict__ a, double (&val)[3]) {
    const int lane = threadIdx.x & 31;
    const int nr = g.ny * g.nz, wpr = (g.nx + 5) >> 2;  // words covering columns 0 .. nx + 1
    const int nw = (int)((gridDim.x * blockDim.x) >> 5);
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    // the sum in FP64; max and min of FP32 values in FP32 (exact, and off the
    // FP64 pipe, which the sum alone keeps busy), widened at the end
    float mx = -INFINITY, mn = INFINITY;
    auto take = [&](float f, int i) {
        if (i >= 1 && i <= g.nx) {
            val[0] += (double)f;
            mx = fmaxf(mx, f);
            mn = fminf(mn, f);
        }
    };
    for (int rb = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); rb < nr; rb += RG * nw) {
        for (int q0 = 0; q0 < wpr; q0 += 64) {
            float4 v[RG][2];
            bool ok[RG][2];
#pragma unroll
            for (int u = 0; u < RG; ++u) {
                const int r = rb + u * nw;
                const bool rv = r < nr;
                const int rr = rv ? r : rb;
                const float4* w = reinterpret_cast<const float4*>(a + gidx(g, 0, 1 + rr % g.ny, 1 + rr / g.ny));
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int q = q0 + lane + 32 * h;
                    ok[u][h] = rv && q < wpr;
                    v[u][h] = ok[u][h] ? w[q] : zero;
                }
            }
#pragma unroll
            for (int u = 0; u < RG; ++u)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    if (ok[u][h]) {
                        const int i = 4 * (q0 + lane + 32 * h);
                        take(v[u][h].x, i);
                        take(v[u][h].y, i + 1);
                        take(v[u][h].z, i + 2);
                        take(v[u][h].w, i + 3);
                    }
        }
    }
    val[1] = fmax(val[1], (double)mx);
    val[2] = fmin(val[2], (double)mn);
}

__global__ void __launch_bounds__(RED_THREADS, 4) k_red_field_fold(Geom g, const float* __restrict__ a,
                                                                double* partial, unsigned* counter,
                                                                double scale, double* result,
                                                                double* host_alias, int slot) {
    double val[3] = {0.0, -INFINITY, INFINITY};
    const int op[3] = {OP_SUM, OP_MAX, OP_MIN};
    field_words(g, a, val);
    block_reduce_store<3>(val, op, partial);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();  // the partial before the count
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    fold_partials(partial, gridDim.x, 3, OP_SUM, OP_MAX, OP_MIN, POST_SCALE, scale, result);
    if (threadIdx.x == 0) {
        if (host_alias) {
            *host_alias = result[slot];
            __threadfence_system();
        }
        *counter = 0u;
    }
}

cudaError_t reduce_launch(const Geom& g, const ReduceInputs& in, int what, double* d_scratch,
                          double* d_result, cudaStream_t s, double* host_alias, bool* wrote_host) {
    const int nblk = RED_BLOCKS;
    double* part = d_scratch;
    const double ncell = (double)g.nx * g.ny * g.nz;
    if (wrote_host) *wrote_host = false;
    switch (what) {
        case RED_VOLUME:
        case RED_F_MIN:
        case RED_F_MAX: {
            const double vol = (double)g.dx * (double)g.dy * (double)g.dz;
            // result[0] = volume, [1] = max, [2] = min
            unsigned* counter = reinterpret_cast<unsigned*>(d_scratch + 3 * RED_BLOCKS);
            k_red_field_fold<<<nblk, RED_THREADS, 0, s>>>(g, in.F, part, counter, vol, d_result, host_alias,
                                                          reduce_result_slot(what));
            if (wrote_host) *wrote_host = host_alias != nullptr;
            break;
        }
        case RED_DIV_L2:
        case RED_DIV_MAX:
            k_red_div<<<nblk, RED_THREADS, 0, s>>>(g, in.u, in.v, in.w, part);
            k_red_finish<<<1, RED_THREADS, 0, s>>>(part, nblk, 2, OP_SUM, OP_MAX, OP_SUM,
                                                   POST_SQRT, 1.0, d_result);
            break;
        case RED_PRES_RESID: {
            // mean(rhs) into d_result[3], then the residual ratio into d_result[0].
            k_red_field<<<nblk, RED_THREADS, 0, s>>>(g, in.rhs, part);
            k_red_finish<<<1, RED_THREADS, 0, s>>>(part, nblk, 3, OP_SUM, OP_MAX, OP_MIN,
                                                   POST_MEAN, 1.0 / ncell, d_result + 3);
            k_red_resid<<<nblk, RED_THREADS, 0, s>>>(g, in.rhs, in.p, d_result + 3, part);
            k_red_finish<<<1, RED_THREADS, 0, s>>>(part, nblk, 2, OP_SUM, OP_SUM, OP_SUM,
                                                   POST_RATIO, 1.0, d_result);
            break;
        }
        case RED_NONFINITE:
            k_red_nonfinite<<<nblk, RED_THREADS, 0, s>>>(g, in.F, in.u, in.v, in.w, in.p, part);
            k_red_finish<<<1, RED_THREADS, 0, s>>>(part, nblk, 1, OP_SUM, OP_SUM, OP_SUM,
                                                   POST_NONE, 1.0, d_result);
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int reduce_result_slot(int what) {
    switch (what) {
        case RED_F_MAX: return 1;
        case RED_F_MIN: return 2;
        case RED_DIV_MAX: return 1;
        default: return 0;
    }
}

}  // namespace vof
