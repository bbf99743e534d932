// mg_solve.cu -- convergent pressure solve for VOF_MODE_MIXED / VOF_MODE_FP64
// (extension of the reference's 10 Jacobi sweeps, voftrial1.cu:401-439,
// 1371-1375; no counterpart in the reference).
//
// System: the reference's Neumann operator A (Sigma over non-wall neighbours
// of (p_nb - p)/h^2) with the right-hand side b = rhs - mean(rhs), which makes
// the singular system consistent; the gauge is fixed by mean(p) = 0.
//
// Outer loop (FP64): defect correction.  r = b - A p in FP64; stop when
// ||r|| <= tol ||b||; otherwise one multigrid V-cycle approximates A e = r
// in the inner precision and p += e in FP64.  The inner solve:
//   MIXED: every multigrid vector stored in BF16, arithmetic in FP32;
//   FP64:  the same cycle with FP64 storage and arithmetic (the yardstick).
// V-cycle: Chebyshev-accelerated Jacobi (the Jacobi update of the reference's
// sweep inside the Chebyshev three-term recurrence) as the smoother, degree 3
// before and after on levels wider than 25 cells (eigenvalues of D^-1 A in
// [1/3, 2]) and degree 8 on smaller ones ([1/15, 2]), averaging restriction, cell-centred
// multilinear prolongation with zero-gradient ends, coarse operators
// rediscretised at the coarse spacing.  Each axis is coarsened by its
// smallest prime factor (2, 3, 5, 7) while at least two cells remain
// (200 -> 100 -> 50 -> 25 -> 5).  The coarsest level is solved exactly with
// a stored inverse of A + c 11^T (mean-free right-hand side) when it has at
// most MG_DENSE_MAX cells, otherwise by 100 damped Jacobi sweeps (omega =
// 6/7) after removing the mean of its right-hand side.
//
// Execution: the large levels run as multi-block kernels (blocks of 32 x 8
// columns marching kc planes, the z neighbours kept in registers); the first
// sweep from zero is fused into the kernel producing the level's right-hand
// side (the FP64 residual, or the restriction), and the last post-sweep of
// the fine level is fused with p += e.  The deepest levels of at most
// MG_TAIL_CELLS cells whose vectors fit in shared memory (with the coarse
// inverse; 5^3 at 200^3) run in one 1024-thread block entirely from shared
// memory (k_mg_tail), which removes the launch-latency floor of the coarse
// levels; one outer iteration is a captured CUDA graph.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>

#include <utility>
#include <vector>

#include "mg_solve.h"

namespace vof {

template <typename S>
struct St;
template <>
struct St<__nv_bfloat16> {
    using C = float;
    __device__ static float ld(const __nv_bfloat16* p, int i) { return __bfloat162float(p[i]); }
    __device__ static void st(__nv_bfloat16* p, int i, float v) { p[i] = __float2bfloat16_rn(v); }
    __device__ static float q(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }
};
template <>
struct St<double> {
    using C = double;
    __device__ static double ld(const double* p, int i) { return p[i]; }
    __device__ static void st(double* p, int i, double v) { p[i] = v; }
    __device__ static double q(double v) { return v; }
};

constexpr int MG_THREADS = MG_BX * MG_BY;
constexpr int TAIL_THREADS = 1024;

// Programmatic dependent launch.  Every kernel of the solve is launched with
// cudaLaunchAttributeProgrammaticStreamSerialization (pdl_launch) and begins
// with pdl_enter(): it waits for the grid before it to complete (and its
// writes to be visible) before its first global memory access, then lets the
// next grid launch.  The launch and prologue of a kernel so overlap the end of
// the one before, which removes most of the gap between the short kernels of
// the coarse levels.  Launched without the attribute, the wait returns at once.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
static cudaError_t pdl_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

__host__ __device__ __forceinline__ int nb_count(int x, int n) { return (x > 0) + (x < n - 1); }

// Sigma over the x/y non-wall neighbours of a (e_nb - ec) at compact index c.
template <typename S, typename C>
__device__ __forceinline__ C lap_xy(const MgLevel& L, const S* e, int c, int i, int j, C ec) {
    using T = St<S>;
    const C ax = (C)L.ax, ay = (C)L.ay;
    C s = 0;
    if (i > 0) s += ax * ((C)T::ld(e, c - 1) - ec);
    if (i < L.nx - 1) s += ax * ((C)T::ld(e, c + 1) - ec);
    if (j > 0) s += ay * ((C)T::ld(e, c - L.nx) - ec);
    if (j < L.ny - 1) s += ay * ((C)T::ld(e, c + L.nx) - ec);
    return s;
}

template <typename C>
__device__ __forceinline__ C lap_z(const MgLevel& L, int k, C ec, C em, C ep) {
    const C az = (C)L.az;
    C s = 0;
    if (k > 0) s += az * (em - ec);
    if (k < L.nz - 1) s += az * (ep - ec);
    return s;
}

// One smoothing step on column (i, j), planes [k0, k1):
//   eout = ein + alpha (ein - xprev) + beta D^-1 (b - mb - A ein),
// xprev = the value eout holds on entry (read_prev) or 0; ein == nullptr
// means ein = 0.
template <typename S>
__device__ __forceinline__ void column_sweep(const MgLevel& L, const S* __restrict__ ein, S* __restrict__ eout,
                                             const S* __restrict__ b, typename St<S>::C mb, typename St<S>::C alpha,
                                             typename St<S>::C beta, bool read_prev, int i, int j, int k0, int k1) {
    using T = St<S>;
    using C = typename T::C;
    const int plane = L.nx * L.ny;
    const int nbxy = nb_count(i, L.nx) * 9 + nb_count(j, L.ny) * 3;
    int c = (k0 * L.ny + j) * L.nx + i;
    C em = 0, ec = 0;
    if (ein) {
        em = k0 > 0 ? (C)T::ld(ein, c - plane) : (C)0;
        ec = (C)T::ld(ein, c);
    }
    for (int k = k0; k < k1; ++k, c += plane) {
        C ep = 0, Ae = 0;
        if (ein) {
            ep = k + 1 < L.nz ? (C)T::ld(ein, c + plane) : (C)0;
            Ae = lap_xy<S, C>(L, ein, c, i, j, ec) + lap_z<C>(L, k, ec, em, ep);
        }
        const C xp = read_prev ? (C)T::ld(eout, c) : (C)0;
        T::st(eout, c, ec + alpha * (ec - xp) + beta * (C)L.idg[nbxy + nb_count(k, L.nz)] * ((C)T::ld(b, c) - mb - Ae));
        em = ec;
        ec = ep;
    }
}

// (b - A e) at compact cell (i, j, k), all neighbours loaded.
template <typename S>
__device__ __forceinline__ typename St<S>::C cell_residual(const MgLevel& L, const S* e, const S* b, int i, int j,
                                                           int k) {
    using T = St<S>;
    using C = typename T::C;
    const int plane = L.nx * L.ny;
    const int c = (k * L.ny + j) * L.nx + i;
    const C ec = (C)T::ld(e, c);
    const C em = k > 0 ? (C)T::ld(e, c - plane) : (C)0;
    const C ep = k < L.nz - 1 ? (C)T::ld(e, c + plane) : (C)0;
    return (C)T::ld(b, c) - (lap_xy<S, C>(L, e, c, i, j, ec) + lap_z<C>(L, k, ec, em, ep));
}

// Cell-centred linear interpolation along one axis: fine cell x of a level
// coarsened by r; the two coarse indices and the weight of hi.
template <typename C>
__device__ __forceinline__ void lin1(int x, int r, int nc, int& lo, int& hi, C& t) {
    if (r == 1) {
        lo = hi = x;
        t = 0;
        return;
    }
    if (r == 2) {  // centre offsets -1/4 and +1/4 of a coarse cell
        const int I = x >> 1;
        lo = (x & 1) ? I : I - 1;
        hi = lo + 1;
        t = (x & 1) ? (C)0.25 : (C)0.75;
        lo = lo < 0 ? 0 : lo;
        hi = hi > nc - 1 ? nc - 1 : hi;
        return;
    }
    const int I = x / r, m = x - I * r;
    const C off = ((C)m + (C)0.5) / (C)r - (C)0.5;  // from the coarse centre, in coarse cells
    if (off < 0) {
        lo = I - 1;
        hi = I;
        t = off + (C)1;
    } else {
        lo = I;
        hi = I + 1;
        t = off;
    }
    lo = lo < 0 ? 0 : lo;
    hi = hi > nc - 1 ? nc - 1 : hi;
}

// e(i,j,k) += (P ec)(i,j,k), multilinear with zero-gradient ends.
template <typename S>
__device__ __forceinline__ void prolong_cell(const MgLevel& F, S* e, const MgLevel& Cl, const S* ec, int i, int j,
                                             int k) {
    using T = St<S>;
    using C = typename T::C;
    int x0, x1, y0, y1, z0, z1;
    C tx, ty, tz;
    lin1<C>(i, F.rx, Cl.nx, x0, x1, tx);
    lin1<C>(j, F.ry, Cl.ny, y0, y1, ty);
    lin1<C>(k, F.rz, Cl.nz, z0, z1, tz);
    const int cp = Cl.nx * Cl.ny;
    const int r00 = z0 * cp + y0 * Cl.nx, r10 = z0 * cp + y1 * Cl.nx;
    const int r01 = z1 * cp + y0 * Cl.nx, r11 = z1 * cp + y1 * Cl.nx;
    const C c00 = (C)T::ld(ec, r00 + x0) * (1 - tx) + (C)T::ld(ec, r00 + x1) * tx;
    const C c10 = (C)T::ld(ec, r10 + x0) * (1 - tx) + (C)T::ld(ec, r10 + x1) * tx;
    const C c01 = (C)T::ld(ec, r01 + x0) * (1 - tx) + (C)T::ld(ec, r01 + x1) * tx;
    const C c11 = (C)T::ld(ec, r11 + x0) * (1 - tx) + (C)T::ld(ec, r11 + x1) * tx;
    const C v = (c00 * (1 - ty) + c10 * ty) * (1 - tz) + (c01 * (1 - ty) + c11 * ty) * tz;
    const int c = (k * F.ny + j) * F.nx + i;
    T::st(e, c, (C)T::ld(e, c) + v);
}

// ---- reductions ---------------------------------------------------------------
// Deterministic block sum of two doubles (block size a multiple of 32, up to
// 1024); every thread gets the totals.
__device__ __forceinline__ void block_sum2(double& a, double& b) {
    __shared__ double sh[2][32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    __syncthreads();  // sh may still be read by a previous call
    if ((tid & 31) == 0) {
        sh[0][tid >> 5] = a;
        sh[1][tid >> 5] = b;
    }
    __syncthreads();
    double x = 0, y = 0;
    for (int q = 0; q < nthr / 32; ++q) {
        x += sh[0][q];
        y += sh[1][q];
    }
    a = x;
    b = y;
}

__device__ __forceinline__ int block_linear() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }

__global__ void __launch_bounds__(MG_THREADS) k_fold2(const double* __restrict__ partial, int nblk,
                                                      double* __restrict__ out, double* host_out) {
    pdl_enter();
    double a = 0, b = 0;
    for (int q = threadIdx.x; q < nblk; q += blockDim.x) {
        a += partial[2 * q];
        b += partial[2 * q + 1];
    }
    block_sum2(a, b);
    if (threadIdx.x == 0) {
        out[0] = a;
        out[1] = b;
        if (host_out) {
            host_out[0] = a;
            host_out[1] = b;
            __threadfence_system();
        }
    }
}

#define LEVEL_TILE(L)                                  \
    const int i = blockIdx.x * MG_BX + threadIdx.x;    \
    const int j = blockIdx.y * MG_BY + threadIdx.y;    \
    const int k0 = blockIdx.z * (L).kc;                \
    const int k1 = min((L).nz, k0 + (L).kc);           \
    const bool active = i < (L).nx && j < (L).ny

// ---- multi-block level kernels ---------------------------------------------------
template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_mg_smooth(MgLevel L, const S* __restrict__ ein,
                                                          S* __restrict__ eout, const S* __restrict__ b,
                                                          const double* __restrict__ bsum, double alpha, double beta,
                                                          int read_prev) {
    pdl_enter();
    using C = typename St<S>::C;
    LEVEL_TILE(L);
    if (!active) return;
    const C mb = bsum ? (C)(bsum[0] / L.ncell) : (C)0;
    column_sweep<S>(L, ein, eout, b, mb, (C)alpha, (C)beta, read_prev != 0, i, j, k0, k1);
}

// The same step for BF16 levels of even width, two cells of a row per thread
// (bf16x2 loads and stores; the x neighbours of a pair come from the
// neighbouring lanes).  Same arithmetic, same order as column_sweep.
__device__ __forceinline__ float2 ld2(const __nv_bfloat16* p, int i) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p + i));
}
__global__ void __launch_bounds__(MG_THREADS) k_mg_smooth2(MgLevel L, const __nv_bfloat16* __restrict__ ein,
                                                           __nv_bfloat16* __restrict__ eout,
                                                           const __nv_bfloat16* __restrict__ b, double alpha_d,
                                                           double beta_d, int read_prev) {
    pdl_enter();
    const int pi = blockIdx.x * MG_BX + threadIdx.x;  // pair index along x
    const int i0 = 2 * pi;
    const int j = blockIdx.y * MG_BY + threadIdx.y;
    const int k0 = blockIdx.z * L.kc;
    const int k1 = min(L.nz, k0 + L.kc);
    const bool act = i0 < L.nx && j < L.ny;
    const int ic = act ? i0 : 0, jc = j < L.ny ? j : 0;  // inactive lanes read a valid pair
    const int plane = L.nx * L.ny;
    const float alpha = (float)alpha_d, beta = (float)beta_d;
    const float ax = (float)L.ax, ay = (float)L.ay, az = (float)L.az;
    const int nby = nb_count(jc, L.ny) * 3;
    const int nb0 = nb_count(ic, L.nx) * 9 + nby, nb1 = nb_count(ic + 1, L.nx) * 9 + nby;
    int c = (k0 * L.ny + jc) * L.nx + ic;
    float2 em = k0 > 0 ? ld2(ein, c - plane) : make_float2(0.0f, 0.0f);
    float2 ec = ld2(ein, c);
    for (int k = k0; k < k1; ++k, c += plane) {
        const float2 ep = k + 1 < L.nz ? ld2(ein, c + plane) : make_float2(0.0f, 0.0f);
        float w = __shfl_up_sync(0xffffffffu, ec.y, 1);    // e(i0 - 1)
        float e2 = __shfl_down_sync(0xffffffffu, ec.x, 1); // e(i0 + 2)
        if (threadIdx.x == 0 && ic > 0) w = __bfloat162float(ein[c - 1]);
        if (threadIdx.x == MG_BX - 1 && ic + 2 < L.nx) e2 = __bfloat162float(ein[c + 2]);
        const float2 sv = jc > 0 ? ld2(ein, c - L.nx) : make_float2(0.0f, 0.0f);
        const float2 nv = jc < L.ny - 1 ? ld2(ein, c + L.nx) : make_float2(0.0f, 0.0f);
        const float2 bv = ld2(b, c);
        const float2 xp = read_prev ? ld2(eout, c) : make_float2(0.0f, 0.0f);
        // cell i0: x- (if i0 > 0), x+ (= i0 + 1, always inside: nx even)
        float s0 = 0.0f;
        if (ic > 0) s0 += ax * (w - ec.x);
        s0 += ax * (ec.y - ec.x);
        if (jc > 0) s0 += ay * (sv.x - ec.x);
        if (jc < L.ny - 1) s0 += ay * (nv.x - ec.x);
        float z0 = 0.0f;
        if (k > 0) z0 += az * (em.x - ec.x);
        if (k < L.nz - 1) z0 += az * (ep.x - ec.x);
        // cell i0 + 1: x- (= i0, always), x+ (if i0 + 2 < nx)
        float s1 = 0.0f;
        s1 += ax * (ec.x - ec.y);
        if (ic + 2 < L.nx) s1 += ax * (e2 - ec.y);
        if (jc > 0) s1 += ay * (sv.y - ec.y);
        if (jc < L.ny - 1) s1 += ay * (nv.y - ec.y);
        float z1 = 0.0f;
        if (k > 0) z1 += az * (em.y - ec.y);
        if (k < L.nz - 1) z1 += az * (ep.y - ec.y);
        const int nbz = nb_count(k, L.nz);
        const float o0 = ec.x + alpha * (ec.x - xp.x) + beta * (float)L.idg[nb0 + nbz] * (bv.x - 0.0f - (s0 + z0));
        const float o1 = ec.y + alpha * (ec.y - xp.y) + beta * (float)L.idg[nb1 + nbz] * (bv.y - 0.0f - (s1 + z1));
        if (act) *reinterpret_cast<__nv_bfloat162*>(eout + c) = __floats2bfloat162_rn(o0, o1);
        em = ec;
        ec = ep;
    }
}

// ---- flat BF16 kernels: two cells per thread, packed FP32 arithmetic ----------
// The cell pairs (i, i + 1), i even, of a level of even width are numbered
// over a plane, p = (j nx + i) / 2, so that a pair is the 32-bit word
// k (nx ny / 2) + p of a BF16 vector.  The flat kernels give 32 consecutive
// pairs (or coarse cells) to a warp across row ends, so every lane has work
// at every width; a thread marches kc planes.  The x neighbours of a pair
// come from the neighbouring lanes (from memory at the ends of a warp), the
// z neighbours stay in registers.  A wall neighbour is replaced by the cell
// itself, which gives at every cell
//   A e = ax (e_w + e_e) + ay (e_s + e_n) + az (e_d + e_u) - 2 (ax + ay + az) e_c,
// evaluated for both cells of a pair at once by the f32x2 instructions of
// sm_100 (add/sub/mul/fma .rn.f32x2: one instruction for the pair).
namespace pk {

__device__ __forceinline__ float2 padd(float2 a, float2 b) {
    float2 r;
    asm("{.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
    float2 r;
    asm("{.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 pmul(float2 a, float2 b) {
    float2 r;
    asm("{.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
// a b + c, one rounding per element
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) {
    float2 r;
    asm("{.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}
__device__ __forceinline__ float2 splat(float a) { return make_float2(a, a); }
// A BF16 pair word to FP32 (first cell in the low half) and back (RN).
__device__ __forceinline__ float2 unpack(unsigned v) {
    return make_float2(__uint_as_float(v << 16), __uint_as_float(v & 0xffff0000u));
}
__device__ __forceinline__ unsigned pack(float2 v) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
    return *reinterpret_cast<const unsigned*>(&h);
}

struct Op {
    float2 ax, ay, az, nd;  // ax, ay, az; nd = -2 (ax + ay + az)
};
__device__ __forceinline__ Op op_of(const MgLevel& L) {
    const float ax = (float)L.ax, ay = (float)L.ay, az = (float)L.az;
    return {splat(ax), splat(ay), splat(az), splat(-2.0f * (ax + ay + az))};
}

// b - A e of a pair with value c, x neighbours xw (of its first cell) and xe
// (of its second), neighbour pairs s, n along y and d, u along z.
__device__ __forceinline__ float2 residual(const Op& o, float2 c, float xw, float xe, float2 s, float2 n, float2 d,
                                           float2 u, float2 b) {
    float2 t = pmul(o.ax, padd(make_float2(xw, c.x), make_float2(c.y, xe)));
    t = pfma(o.ay, padd(s, n), t);
    t = pfma(o.az, padd(d, u), t);
    return psub(b, pfma(o.nd, c, t));
}

// Where a lane's x neighbours come from: hw / he, the pair has a west / east
// neighbour cell; ldw / lde, that neighbour is read from memory (lane 0 / 31).
struct XNb {
    bool hw, he, ldw, lde;
};
__device__ __forceinline__ XNb xnb_of(int ip, int npr) {
    const int lane = threadIdx.x & 31;
    XNb f;
    f.hw = ip > 0;
    f.he = ip < npr - 1;
    f.ldw = f.hw && lane == 0;
    f.lde = f.he && lane == 31;
    return f;
}
// The x neighbours of pair value c whose first cell is the 16-bit element h0
// of h (every lane of the warp calls this).
__device__ __forceinline__ void xnb(float2 c, const unsigned short* __restrict__ h, int h0, const XNb& f, float& xw,
                                   float& xe) {
    xw = __shfl_up_sync(0xffffffffu, c.y, 1);
    xe = __shfl_down_sync(0xffffffffu, c.x, 1);
    if (f.ldw) xw = __uint_as_float((unsigned)__ldg(h + h0 - 1) << 16);
    if (f.lde) xe = __uint_as_float((unsigned)__ldg(h + h0 + 2) << 16);
    if (!f.hw) xw = c.x;
    if (!f.he) xe = c.y;
}

}  // namespace pk

// One Chebyshev smoothing step (as column_sweep with mb = 0) on the pairs of
// an even-width BF16 level; grid (pgx, pgz), pkc planes per block.
template <bool READ_PREV>
__global__ void __launch_bounds__(MG_FLAT_THREADS) k_mg_smooth_pairs(MgLevel L, const unsigned* __restrict__ ein,
                                                                     unsigned* __restrict__ eout,
                                                                     const unsigned* __restrict__ b, float alpha,
                                                                     float beta) {
    pdl_enter();
    using namespace pk;
    const int npr = L.nx >> 1, npl = npr * L.ny;
    const int q0 = blockIdx.x * MG_FLAT_THREADS + threadIdx.x;
    const bool act = q0 < npl;
    const int p = act ? q0 : npl - 1;  // lanes past the end shadow the last pair
    const int j = p / npr, ip = p - j * npr;
    const XNb f = xnb_of(ip, npr);
    const bool hs = j > 0, hn = j < L.ny - 1;
    const int k0 = blockIdx.y * L.pkc, k1 = min(L.nz, k0 + L.pkc);
    const Op op = op_of(L);
    // beta / diag(A) of the two cells on inner planes and on the end planes
    const int nby = ((int)hs + (int)hn) * 3;
    const int n0 = ((int)f.hw + 1) * 9 + nby, n1 = (1 + (int)f.he) * 9 + nby;
    const int ze = L.nz > 1 ? 1 : 0;
    const float2 bmid = make_float2(beta * (float)L.idg[n0 + 2], beta * (float)L.idg[n1 + 2]);
    const float2 bend = make_float2(beta * (float)L.idg[n0 + ze], beta * (float)L.idg[n1 + ze]);
    const float2 al = splat(alpha);
    const unsigned short* h = reinterpret_cast<const unsigned short*>(ein);
    int w = k0 * npl + p;
    float2 ec = unpack(__ldg(ein + w));
    float2 ed = k0 > 0 ? unpack(__ldg(ein + w - npl)) : ec;
    for (int k = k0; k < k1; ++k, w += npl) {
        const float2 eu = k + 1 < L.nz ? unpack(__ldg(ein + w + npl)) : ec;
        const float2 es = hs ? unpack(__ldg(ein + w - npr)) : ec;
        const float2 en = hn ? unpack(__ldg(ein + w + npr)) : ec;
        float xw, xe;
        xnb(ec, h, 2 * w, f, xw, xe);
        const float2 r = residual(op, ec, xw, xe, es, en, ed, eu, unpack(__ldg(b + w)));
        const float2 xp = READ_PREV ? unpack(eout[w]) : make_float2(0.0f, 0.0f);
        const float2 o = pfma((k == 0 || k == L.nz - 1) ? bend : bmid, r, pfma(al, psub(ec, xp), ec));
        if (act) eout[w] = pack(o);
        ed = ec;
        ec = eu;
    }
}

// Coarse right-hand side of a 2 x 2 x 2 coarsening of an even-width BF16
// level F: one thread per coarse column (I, J), flat over the coarse plane
// (grid (cgx, cgz) of the coarse level, ckc planes per block).  Per coarse
// plane K the thread sums the fine residuals of the pairs (2I, 2I + 1) in rows
// 2J, 2J + 1 of planes 2K, 2K + 1 (rows 2J - 1 .. 2J + 2 read, the planes
// below and above kept in registers); ec (optional) = the first smoothing
// step from zero at the coarse level.
__global__ void __launch_bounds__(MG_FLAT_THREADS) k_mg_restrict_pairs(MgLevel F, const unsigned* __restrict__ e,
                                                                       const unsigned* __restrict__ b, MgLevel Cl,
                                                                       __nv_bfloat16* __restrict__ bc,
                                                                       __nv_bfloat16* __restrict__ ec) {
    pdl_enter();
    using namespace pk;
    const int cn = Cl.nx * Cl.ny;
    const int q0 = blockIdx.x * MG_FLAT_THREADS + threadIdx.x;
    const bool act = q0 < cn;
    const int q = act ? q0 : cn - 1;
    const int J = q / Cl.nx, I = q - J * Cl.nx;
    const XNb f = xnb_of(I, Cl.nx);  // the fine pairs of a row number I = 0 .. Cl.nx - 1
    const bool hs = J > 0, hn = J < Cl.ny - 1;
    const int K0 = blockIdx.y * Cl.ckc, K1 = min(Cl.nz, K0 + Cl.ckc);
    const Op op = op_of(F);
    const int npr = F.nx >> 1, npl = npr * F.ny;  // fine pairs per row, per plane
    const unsigned short* h = reinterpret_cast<const unsigned short*>(e);
    const int nbxy = nb_count(I, Cl.nx) * 9 + nb_count(J, Cl.ny) * 3;
    const float cb0 = (float)Cl.cb[0];
    int w = 2 * K0 * npl + 2 * J * npr + I;  // pair of fine row 2J, plane 2K
    // rows 2J, 2J + 1 of fine plane 2K - 1 (plane 2K itself at the bottom wall)
    const int wd = K0 > 0 ? w - npl : w;
    float2 da = unpack(__ldg(e + wd)), db = unpack(__ldg(e + wd + npr));
    for (int K = K0; K < K1; ++K, w += 2 * npl) {
        const int w1 = w + npl;  // plane 2K + 1
        const float2 a0 = unpack(__ldg(e + w)), b0 = unpack(__ldg(e + w + npr));
        const float2 s0 = hs ? unpack(__ldg(e + w - npr)) : a0;
        const float2 n0 = hn ? unpack(__ldg(e + w + 2 * npr)) : b0;
        const float2 a1 = unpack(__ldg(e + w1)), b1 = unpack(__ldg(e + w1 + npr));
        const float2 s1 = hs ? unpack(__ldg(e + w1 - npr)) : a1;
        const float2 n1 = hn ? unpack(__ldg(e + w1 + 2 * npr)) : b1;
        // rows 2J, 2J + 1 of plane 2K + 2 (plane 2K + 1 itself at the top wall)
        const bool up = K + 1 < Cl.nz;
        const float2 ua = up ? unpack(__ldg(e + w1 + npl)) : a1;
        const float2 ub = up ? unpack(__ldg(e + w1 + npl + npr)) : b1;
        float xw, xe;
        xnb(a0, h, 2 * w, f, xw, xe);
        float2 acc = residual(op, a0, xw, xe, s0, b0, da, a1, unpack(__ldg(b + w)));
        xnb(b0, h, 2 * (w + npr), f, xw, xe);
        acc = padd(acc, residual(op, b0, xw, xe, a0, n0, db, b1, unpack(__ldg(b + w + npr))));
        xnb(a1, h, 2 * w1, f, xw, xe);
        acc = padd(acc, residual(op, a1, xw, xe, s1, b1, a0, ua, unpack(__ldg(b + w1))));
        xnb(b1, h, 2 * (w1 + npr), f, xw, xe);
        acc = padd(acc, residual(op, b1, xw, xe, a1, n1, b0, ub, unpack(__ldg(b + w1 + npr))));
        if (act) {
            const int c = K * cn + q;
            const __nv_bfloat16 v = __float2bfloat16_rn((acc.x + acc.y) * 0.125f);
            bc[c] = v;
            if (ec)
                ec[c] = __float2bfloat16_rn(cb0 * (float)Cl.idg[nbxy + nb_count(K, Cl.nz)] * __bfloat162float(v));
        }
        da = a1;
        db = b1;
    }
}

// e += P ec for a 2 x 2 x 2 coarsening of an even-width BF16 level F: one
// thread per coarse column (I, J) (grid (cgx, cgz) of the coarse level),
// marching the coarse planes; per coarse plane K it adds the trilinear
// interpolant (weights 3/4 and 1/4 along each axis, the coarse index clamped
// at the ends: zero gradient) to the fine pairs (2I, 2I + 1) of rows 2J,
// 2J + 1 in planes 2K, 2K + 1.
__global__ void __launch_bounds__(MG_FLAT_THREADS) k_mg_prolong_pairs(MgLevel F, unsigned* __restrict__ e,
                                                                      MgLevel Cl,
                                                                      const __nv_bfloat16* __restrict__ ecrs) {
    pdl_enter();
    using namespace pk;
    const int cn = Cl.nx * Cl.ny;
    const int q0 = blockIdx.x * MG_FLAT_THREADS + threadIdx.x;
    const bool act = q0 < cn;
    const int q = act ? q0 : cn - 1;
    const int J = q / Cl.nx, I = q - J * Cl.nx;
    const XNb f = xnb_of(I, Cl.nx);
    const int dS = J > 0 ? -Cl.nx : 0, dN = J < Cl.ny - 1 ? Cl.nx : 0;  // coarse rows J -/+ 1, clamped
    const int K0 = blockIdx.y * Cl.ckc, K1 = min(Cl.nz, K0 + Cl.ckc);
    const int npr = F.nx >> 1, npl = npr * F.ny;
    const float2 w1 = splat(0.25f), w3 = splat(0.75f);
    // x interpolation of the coarse row holding element c: values at fine 2I, 2I + 1
    auto xrow = [&](int c) -> float2 {
        const float v = __bfloat162float(__ldg(ecrs + c));
        float vw = __shfl_up_sync(0xffffffffu, v, 1), ve = __shfl_down_sync(0xffffffffu, v, 1);
        if (f.ldw) vw = __bfloat162float(__ldg(ecrs + c - 1));
        if (f.lde) ve = __bfloat162float(__ldg(ecrs + c + 1));
        if (!f.hw) vw = v;
        if (!f.he) ve = v;
        return pfma(w3, splat(v), pmul(w1, make_float2(vw, ve)));
    };
    // fine rows 2J (from J - 1, J) and 2J + 1 (from J, J + 1) of coarse plane K
    auto yplane = [&](int K, float2& r0, float2& r1) {
        const int c = K * cn + q;
        const float2 xs = xrow(c + dS), xc = xrow(c), xn = xrow(c + dN);
        r0 = pfma(w3, xc, pmul(w1, xs));
        r1 = pfma(w3, xc, pmul(w1, xn));
    };
    float2 d0, d1, c0, c1;  // coarse planes K - 1 (clamped) and K
    yplane(K0 > 0 ? K0 - 1 : 0, d0, d1);
    yplane(K0, c0, c1);
    int w = 2 * K0 * npl + 2 * J * npr + I;
    for (int K = K0; K < K1; ++K, w += 2 * npl) {
        float2 u0, u1;
        yplane(K + 1 < Cl.nz ? K + 1 : K, u0, u1);
        if (act) {
            const int ws[4] = {w, w + npr, w + npl, w + npl + npr};
            const float2 v[4] = {pfma(w3, c0, pmul(w1, d0)), pfma(w3, c1, pmul(w1, d1)), pfma(w3, c0, pmul(w1, u0)),
                                 pfma(w3, c1, pmul(w1, u1))};
#pragma unroll
            for (int t = 0; t < 4; ++t) e[ws[t]] = pack(padd(unpack(e[ws[t]]), v[t]));
        }
        d0 = c0;
        d1 = c1;
        c0 = u0;
        c1 = u1;
    }
}

// Coarse right-hand side = average of the fine residual over each coarse
// cell; ec (optional) = the first smoothing step from zero at the coarse level.
template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_mg_restrict(MgLevel F, const S* __restrict__ e,
                                                            const S* __restrict__ b, MgLevel Cl,
                                                            S* __restrict__ bc, S* __restrict__ ec) {
    pdl_enter();
    using T = St<S>;
    using C = typename T::C;
    LEVEL_TILE(Cl);
    if (!active) return;
    const C inv = (C)(1.0 / (F.rx * F.ry * F.rz));
    const int nbxy = nb_count(i, Cl.nx) * 9 + nb_count(j, Cl.ny) * 3;
    for (int K = k0; K < k1; ++K) {
        C acc = 0;
        for (int dk = 0; dk < F.rz; ++dk)
            for (int dj = 0; dj < F.ry; ++dj)
                for (int di = 0; di < F.rx; ++di)
                    acc += cell_residual<S>(F, e, b, i * F.rx + di, j * F.ry + dj, K * F.rz + dk);
        const C v = acc * inv;
        const int c = (K * Cl.ny + j) * Cl.nx + i;
        T::st(bc, c, v);
        if (ec) T::st(ec, c, (C)Cl.cb[0] * (C)Cl.idg[nbxy + nb_count(K, Cl.nz)] * T::q(v));
    }
}

// The same for coarsening ratios above 8 cells per coarse cell (3, 5, 7 along
// an axis): one block of RW_THREADS per coarse cell sums its fine residuals.
constexpr int RW_THREADS = 128;
template <typename S>
__global__ void __launch_bounds__(RW_THREADS) k_mg_restrict_wide(MgLevel F, const S* __restrict__ e,
                                                                 const S* __restrict__ b, MgLevel Cl,
                                                                 S* __restrict__ bc, S* __restrict__ ec) {
    pdl_enter();
    using T = St<S>;
    using C = typename T::C;
    __shared__ C part[RW_THREADS / 32];
    const int c = blockIdx.x;
    const int I = c % Cl.nx, J = (c / Cl.nx) % Cl.ny, K = c / (Cl.nx * Cl.ny);
    const int nf = F.rx * F.ry * F.rz;
    C acc = 0;
    for (int t = threadIdx.x; t < nf; t += RW_THREADS) {
        const int di = t % F.rx, dj = (t / F.rx) % F.ry, dk = t / (F.rx * F.ry);
        acc += cell_residual<S>(F, e, b, I * F.rx + di, J * F.ry + dj, K * F.rz + dk);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        C sum = 0;
        for (int q = 0; q < RW_THREADS / 32; ++q) sum += part[q];
        const C v = sum * (C)(1.0 / nf);
        T::st(bc, c, v);
        if (ec)
            T::st(ec, c, (C)Cl.cb[0] * (C)Cl.idg[nb_count(I, Cl.nx) * 9 + nb_count(J, Cl.ny) * 3 + nb_count(K, Cl.nz)] *
                             T::q(v));
    }
}

template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_mg_prolong(MgLevel F, S* __restrict__ e, MgLevel Cl,
                                                           const S* __restrict__ ec) {
    pdl_enter();
    LEVEL_TILE(F);
    if (!active) return;
    for (int k = k0; k < k1; ++k) prolong_cell<S>(F, e, Cl, ec, i, j, k);
}

template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_level_sum(MgLevel L, const S* __restrict__ b,
                                                          double* __restrict__ partial) {
    pdl_enter();
    LEVEL_TILE(L);
    double a = 0, z = 0;
    if (active)
        for (int k = k0; k < k1; ++k) a += (double)St<S>::ld(b, (k * L.ny + j) * L.nx + i);
    block_sum2(a, z);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        partial[2 * block_linear()] = a;
        partial[2 * block_linear() + 1] = 0.0;
    }
}

// ---- fine level, FP64 (padded layout of the step) ----------------------------------
template <typename R>
__global__ void __launch_bounds__(MG_THREADS) k_sum_rhs(Geom g, MgLevel L0, const R* __restrict__ rhs,
                                                        double* __restrict__ partial) {
    pdl_enter();
    LEVEL_TILE(L0);
    double a = 0, z = 0;
    if (active)
        for (int k = k0; k < k1; ++k) a += (double)rhs[gidx(g, i + 1, j + 1, k + 1)];
    block_sum2(a, z);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        partial[2 * block_linear()] = a;
        partial[2 * block_linear() + 1] = 0.0;
    }
}

// r = (rhs - mean) - A p in FP64, stored as the fine right-hand side b0;
// e0 (optional) = the first smoothing step from zero; partial sums of r^2, b^2.
template <typename S, typename R>
__global__ void __launch_bounds__(MG_THREADS) k_resid0(Geom g, MgLevel L0, const R* __restrict__ rhs,
                                                       const double* __restrict__ sums, const double* __restrict__ p,
                                                       S* __restrict__ b0, S* __restrict__ e0,
                                                       double* __restrict__ partial) {
    pdl_enter();
    using T = St<S>;
    using C = typename T::C;
    LEVEL_TILE(L0);
    double rr = 0, bb = 0;
    if (active) {
        const double mean = sums[0] / (double)L0.ncell;
        const double ax = L0.ax, ay = L0.ay, az = L0.az;
        const int nbxy = nb_count(i, L0.nx) * 9 + nb_count(j, L0.ny) * 3;
        const int cplane = L0.nx * L0.ny;
        int id = gidx(g, i + 1, j + 1, k0 + 1);
        int c = (k0 * L0.ny + j) * L0.nx + i;
        double pm = k0 > 0 ? p[id - g.plane] : 0.0, pc = p[id];
        for (int k = k0; k < k1; ++k, id += g.plane, c += cplane) {
            const double pp = k + 1 < L0.nz ? p[id + g.plane] : 0.0;
            double s = 0;
            if (i > 0) s += ax * (p[id - 1] - pc);
            if (i < L0.nx - 1) s += ax * (p[id + 1] - pc);
            if (j > 0) s += ay * (p[id - g.px] - pc);
            if (j < L0.ny - 1) s += ay * (p[id + g.px] - pc);
            if (k > 0) s += az * (pm - pc);
            if (k < L0.nz - 1) s += az * (pp - pc);
            const double b = (double)rhs[id] - mean;
            const double r = b - s;
            rr += r * r;
            bb += b * b;
            T::st(b0, c, (C)r);
            if (e0) T::st(e0, c, (C)L0.cb[0] * (C)L0.idg[nbxy + nb_count(k, L0.nz)] * T::q((C)r));
            pm = pc;
            pc = pp;
        }
    }
    block_sum2(rr, bb);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        partial[2 * block_linear()] = rr;
        partial[2 * block_linear() + 1] = bb;
    }
}

// Last post-smoothing step of the fine level fused with p += e (xprev read
// from `prev` when read_prev).
template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_smooth_update(Geom g, MgLevel L0, const S* __restrict__ ein,
                                                              const S* __restrict__ prev, const S* __restrict__ b,
                                                              double* __restrict__ p, double alpha, double beta,
                                                              int read_prev) {
    pdl_enter();
    using T = St<S>;
    using C = typename T::C;
    LEVEL_TILE(L0);
    if (!active) return;
    const int plane = L0.nx * L0.ny;
    const int nbxy = nb_count(i, L0.nx) * 9 + nb_count(j, L0.ny) * 3;
    int c = (k0 * L0.ny + j) * L0.nx + i;
    int id = gidx(g, i + 1, j + 1, k0 + 1);
    C em = k0 > 0 ? (C)T::ld(ein, c - plane) : (C)0, ec = (C)T::ld(ein, c);
    for (int k = k0; k < k1; ++k, c += plane, id += g.plane) {
        const C ep = k + 1 < L0.nz ? (C)T::ld(ein, c + plane) : (C)0;
        const C Ae = lap_xy<S, C>(L0, ein, c, i, j, ec) + lap_z<C>(L0, k, ec, em, ep);
        const C xp = read_prev ? (C)T::ld(prev, c) : (C)0;
        const C en = ec + (C)alpha * (ec - xp) + (C)beta * (C)L0.idg[nbxy + nb_count(k, L0.nz)] * ((C)T::ld(b, c) - Ae);
        p[id] += (double)T::q(en);
        em = ec;
        ec = ep;
    }
}

// p += e (the fine level solved entirely by the one-block kernel).
template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_update64(Geom g, MgLevel L0, double* __restrict__ p,
                                                         const S* __restrict__ e) {
    pdl_enter();
    LEVEL_TILE(L0);
    if (!active) return;
    for (int k = k0; k < k1; ++k) p[gidx(g, i + 1, j + 1, k + 1)] += (double)St<S>::ld(e, (k * L0.ny + j) * L0.nx + i);
}

__global__ void __launch_bounds__(MG_THREADS) k_sum_p(Geom g, MgLevel L0, const double* __restrict__ p,
                                                      double* __restrict__ partial) {
    pdl_enter();
    LEVEL_TILE(L0);
    double a = 0, z = 0;
    if (active)
        for (int k = k0; k < k1; ++k) a += p[gidx(g, i + 1, j + 1, k + 1)];
    block_sum2(a, z);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        partial[2 * block_linear()] = a;
        partial[2 * block_linear() + 1] = 0.0;
    }
}

// p -= mean(p) (gauge), p32 = float(p) on the interior.
__global__ void __launch_bounds__(MG_THREADS) k_gauge_cast(Geom g, MgLevel L0, double* __restrict__ p,
                                                           const double* __restrict__ sump, float* __restrict__ p32) {
    pdl_enter();
    LEVEL_TILE(L0);
    if (!active) return;
    const double mean = sump[0] / (double)L0.ncell;
    for (int k = k0; k < k1; ++k) {
        const int id = gidx(g, i + 1, j + 1, k + 1);
        const double v = p[id] - mean;
        p[id] = v;
        if (p32) p32[id] = (float)v;
    }
}

__global__ void __launch_bounds__(MG_THREADS) k_widen(Geom g, MgLevel L0, const float* __restrict__ p32,
                                                      double* __restrict__ p) {
    pdl_enter();
    LEVEL_TILE(L0);
    if (!active) return;
    for (int k = k0; k < k1; ++k) {
        const int id = gidx(g, i + 1, j + 1, k + 1);
        p[id] = (double)p32[id];
    }
}

// ---- small levels: one block --------------------------------------------------------
// Levels lv[0 .. nl-1] (the last is the coarsest) of one V-cycle after b of
// lv[0] has been written to global memory.  Every vector of these levels
// (and the dense coarse inverse) lives in shared memory for the whole
// kernel; b of lv[0] is read from global memory at the start and the final
// correction of lv[0] written back to `out` at the end.
template <typename S>
__device__ void tail_sweep(const MgLevel& L, const S* ein, S* eout, const S* b, typename St<S>::C mb,
                           typename St<S>::C alpha, typename St<S>::C beta, bool read_prev) {
    for (int j = threadIdx.x >> 5; j < L.ny; j += TAIL_THREADS / 32)
        for (int i = threadIdx.x & 31; i < L.nx; i += 32)
            column_sweep<S>(L, ein, eout, b, mb, alpha, beta, read_prev, i, j, 0, L.nz);
    __syncthreads();
}

template <typename S>
__device__ void tail_restrict(const MgLevel& F, const S* e, const S* b, S* scratch, const MgLevel& Cl) {
    using T = St<S>;
    using C = typename T::C;
    for (int c = threadIdx.x; c < F.ncell; c += TAIL_THREADS) {
        const int i = c % F.nx, j = (c / F.nx) % F.ny, k = c / (F.nx * F.ny);
        T::st(scratch, c, cell_residual<S>(F, e, b, i, j, k));
    }
    __syncthreads();
    const C inv = (C)(1.0 / (F.rx * F.ry * F.rz));
    S* bc = static_cast<S*>(Cl.b);
    for (int c = threadIdx.x; c < Cl.ncell; c += TAIL_THREADS) {
        const int I = c % Cl.nx, J = (c / Cl.nx) % Cl.ny, K = c / (Cl.nx * Cl.ny);
        C acc = 0;
        for (int dk = 0; dk < F.rz; ++dk)
            for (int dj = 0; dj < F.ry; ++dj) {
                const int row = ((K * F.rz + dk) * F.ny + J * F.ry + dj) * F.nx + I * F.rx;
                for (int di = 0; di < F.rx; ++di) acc += (C)T::ld(scratch, row + di);
            }
        T::st(bc, c, acc * inv);
    }
    __syncthreads();
}

template <typename S>
__device__ void tail_prolong(const MgLevel& F, S* e, const MgLevel& Cl, const S* ec) {
    for (int c = threadIdx.x; c < F.ncell; c += TAIL_THREADS) {
        const int i = c % F.nx, j = (c / F.nx) % F.ny, k = c / (F.nx * F.ny);
        prolong_cell<S>(F, e, Cl, ec, i, j, k);
    }
    __syncthreads();
}

template <typename S>
__device__ typename St<S>::C tail_mean(const MgLevel& L, const S* b) {
    double a = 0, z = 0;
    for (int c = threadIdx.x; c < L.ncell; c += TAIL_THREADS) a += (double)St<S>::ld(b, c);
    block_sum2(a, z);
    return (typename St<S>::C)(a / L.ncell);
}

// Bytes of shared memory of one tail vector (16-byte multiple).
__host__ __device__ __forceinline__ int tail_vec_bytes(int ncell, int elem) { return (ncell * elem + 15) & ~15; }

template <typename S>
__global__ void __launch_bounds__(TAIL_THREADS) k_mg_tail(const MgLevel* lv, int nl,
                                                          const typename St<S>::C* cinv_g, S* out) {
    pdl_enter();
    using T = St<S>;
    using C = typename T::C;
    extern __shared__ __align__(16) unsigned char tail_smem[];
    __shared__ MgLevel sl[MG_MAX_LEVELS];
    __shared__ int pre_cur[MG_MAX_LEVELS];
    __shared__ int cinv_off;
    for (int q = threadIdx.x; q < nl * (int)(sizeof(MgLevel) / sizeof(int)); q += TAIL_THREADS)
        reinterpret_cast<int*>(sl)[q] = reinterpret_cast<const int*>(lv)[q];
    __syncthreads();
    const S* b_g = static_cast<const S*>(sl[0].b);
    __syncthreads();
    if (threadIdx.x == 0) {  // re-point every vector into shared memory
        unsigned char* p = tail_smem;
        for (int l = 0; l < nl; ++l) {
            const int vb = tail_vec_bytes(sl[l].ncell, (int)sizeof(S));
            sl[l].e0 = p;
            sl[l].e1 = p + vb;
            sl[l].b = p + 2 * vb;
            p += 3 * vb;
        }
        cinv_off = (int)(p - tail_smem);
    }
    __syncthreads();
    const int last = nl - 1;
    const int nc = sl[last].ncell;
    C* cinv = cinv_g ? reinterpret_cast<C*>(tail_smem + cinv_off) : nullptr;
    {
        S* b0 = static_cast<S*>(sl[0].b);
        for (int c = threadIdx.x; c < sl[0].ncell; c += TAIL_THREADS) b0[c] = b_g[c];
        if (cinv)
            for (int q = threadIdx.x; q < nc * nc; q += TAIL_THREADS) cinv[q] = cinv_g[q];
    }
    __syncthreads();
    for (int l = 0; l < last; ++l) {
        const MgLevel& L = sl[l];
        S* e[2] = {static_cast<S*>(L.e0), static_cast<S*>(L.e1)};
        const S* b = static_cast<const S*>(L.b);
        tail_sweep<S>(L, nullptr, e[0], b, (C)0, (C)0, (C)L.cb[0], false);
        int cur = 0;
        for (int q = 1; q < L.nu; ++q, cur ^= 1)
            tail_sweep<S>(L, e[cur], e[cur ^ 1], b, (C)0, (C)L.ca[q], (C)L.cb[q], q >= 2);
        tail_restrict<S>(L, e[cur], b, e[cur ^ 1], sl[l + 1]);
        if (threadIdx.x == 0) pre_cur[l] = cur;
    }
    {
        const MgLevel& L = sl[last];
        S* e[2] = {static_cast<S*>(L.e0), static_cast<S*>(L.e1)};
        const S* b = static_cast<const S*>(L.b);
        const C mb = tail_mean<S>(L, b);
        if (cinv) {  // e = (A + c 11^T)^-1 (b - mean b); the inverse is symmetric
            for (int c = threadIdx.x; c < nc; c += TAIL_THREADS) {
                C acc = 0;
                for (int q = 0; q < nc; ++q) acc += cinv[q * nc + c] * ((C)T::ld(b, q) - mb);
                T::st(e[0], c, acc);
            }
            __syncthreads();
        } else {
            tail_sweep<S>(L, nullptr, e[0], b, mb, (C)0, (C)MG_OMEGA, false);
            for (int q = 1; q < MG_COARSE_SWEEPS; ++q)
                tail_sweep<S>(L, e[(q - 1) & 1], e[q & 1], b, mb, (C)0, (C)MG_OMEGA, false);
        }
    }
    __syncthreads();
    for (int l = last - 1; l >= 0; --l) {
        const MgLevel& L = sl[l];
        const MgLevel& Cl = sl[l + 1];
        S* e[2] = {static_cast<S*>(L.e0), static_cast<S*>(L.e1)};
        const S* b = static_cast<const S*>(L.b);
        const bool coarse_e0 = (l + 1 == last) && (cinv || !((MG_COARSE_SWEEPS - 1) & 1));
        const S* ec = static_cast<const S*>(coarse_e0 ? Cl.e0 : Cl.e1);
        int cur = pre_cur[l];
        tail_prolong<S>(L, e[cur], Cl, ec);
        for (int q = 0; q < L.nu; ++q, cur ^= 1)
            tail_sweep<S>(L, e[cur], e[cur ^ 1], b, (C)0, (C)L.ca[q], (C)L.cb[q], q >= 1);
    }
    const bool fin_e0 = (last == 0) && (cinv || !((MG_COARSE_SWEEPS - 1) & 1));
    const S* fin = static_cast<const S*>(fin_e0 ? sl[0].e0 : sl[0].e1);
    for (int c = threadIdx.x; c < sl[0].ncell; c += TAIL_THREADS) out[c] = fin[c];
}

// ---- host -------------------------------------------------------------------
static int smallest_factor(int n) {
    const int f[4] = {2, 3, 5, 7};
    for (int q = 0; q < 4; ++q)
        if (n % f[q] == 0 && n / f[q] >= 2) return f[q];
    return 1;
}

// Flat tiling: gx blocks of MG_FLAT_THREADS over `cols` columns of a plane,
// gz blocks of kc planes, about two waves of blocks in all.
static void flat_tiling(int cols, int nz, int& gx, int& gz, int& kc) {
    gx = (cols + MG_FLAT_THREADS - 1) / MG_FLAT_THREADS;
    const int want = 2 * 148 * 8;
    int zc = (want + gx - 1) / gx;
    zc = zc < 1 ? 1 : (zc > nz ? nz : zc);
    kc = (nz + zc - 1) / zc;
    gz = (nz + kc - 1) / kc;
}

static void tiling(MgLevel& m) {
    m.gx = (m.nx + MG_BX - 1) / MG_BX;
    m.gy = (m.ny + MG_BY - 1) / MG_BY;
    const int want = 4 * 148 * 8;  // about four waves of 256-thread blocks
    int zc = (want + m.gx * m.gy - 1) / (m.gx * m.gy);
    zc = zc < 1 ? 1 : (zc > m.nz ? m.nz : zc);
    m.kc = (m.nz + zc - 1) / zc;
    m.gz = (m.nz + m.kc - 1) / m.kc;
    if ((m.nx & 1) == 0)
        flat_tiling(m.nx / 2 * m.ny, m.nz, m.pgx, m.pgz, m.pkc);
    else
        m.pgx = m.pgz = m.pkc = 0;
    flat_tiling(m.nx * m.ny, m.nz, m.cgx, m.cgz, m.ckc);
}

// Coefficients of the Chebyshev smoother of degree nu on [lo, hi] in the
// two-term form x_{q+1} = x_q + ca[q] (x_q - x_{q-1}) + cb[q] D^-1 r_q.
static void chebyshev(int nu, double lo, double hi, double* ca, double* cb) {
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
    double rho = 1.0 / sigma;
    ca[0] = 0.0;
    cb[0] = 1.0 / theta;
    for (int q = 1; q < nu; ++q) {
        const double rn = 1.0 / (2.0 * sigma - rho);
        ca[q] = rn * rho;
        cb[q] = 2.0 * rn / delta;
        rho = rn;
    }
}

int mg_plan(const Geom& g, MgLevel* lv, int max_levels) {
    int n[3] = {g.nx, g.ny, g.nz};
    // level 0 uses the coefficients of the FP64 outer operator: (double)(1/h)^2
    double a[3] = {(double)g.dxi * g.dxi, (double)g.dyi * g.dyi, (double)g.dzi * g.dzi};
    int L = 0;
    while (L < max_levels) {
        MgLevel& m = lv[L];
        m = MgLevel{};
        m.nx = n[0];
        m.ny = n[1];
        m.nz = n[2];
        m.ncell = n[0] * n[1] * n[2];
        m.ax = a[0];
        m.ay = a[1];
        m.az = a[2];
        for (int x = 0; x < 3; ++x)
            for (int y = 0; y < 3; ++y)
                for (int z = 0; z < 3; ++z) {
                    const double d = a[0] * x + a[1] * y + a[2] * z;
                    m.idg[x * 9 + y * 3 + z] = d > 0 ? -1.0 / d : 0.0;
                }
        const bool wide = n[0] > 25 || n[1] > 25 || n[2] > 25;
        m.nu = wide ? MG_NU_FINE : MG_NU_COARSE;
        chebyshev(m.nu, MG_CHEB_HI / (wide ? MG_RATIO_FINE : MG_RATIO_COARSE), MG_CHEB_HI, m.ca, m.cb);
        tiling(m);
        int r[3];
        for (int x = 0; x < 3; ++x) r[x] = (n[x] > 2) ? smallest_factor(n[x]) : 1;
        const bool last = (r[0] == 1 && r[1] == 1 && r[2] == 1) || (n[0] <= 3 && n[1] <= 3 && n[2] <= 3) ||
                          L == max_levels - 1;
        m.rx = last ? 1 : r[0];
        m.ry = last ? 1 : r[1];
        m.rz = last ? 1 : r[2];
        ++L;
        if (last) break;
        for (int x = 0; x < 3; ++x) {
            n[x] /= r[x];
            a[x] /= (double)r[x] * r[x];
        }
    }
    return L;
}

// Inverse of A + c 11^T (c = -(ax+ay+az)/n, nonsingular) of level L by
// Gauss-Jordan elimination with partial pivoting, row-major n x n.
static bool dense_inverse(const MgLevel& L, std::vector<double>& inv) {
    const int n = L.ncell;
    std::vector<double> M((size_t)n * n, 0.0);
    inv.assign((size_t)n * n, 0.0);
    const double c = -(L.ax + L.ay + L.az) / n;
    for (int r = 0; r < n; ++r) {
        for (int q = 0; q < n; ++q) M[(size_t)r * n + q] = c;
        inv[(size_t)r * n + r] = 1.0;
        const int i = r % L.nx, j = (r / L.nx) % L.ny, k = r / (L.nx * L.ny);
        const int has[6] = {i > 0, i < L.nx - 1, j > 0, j < L.ny - 1, k > 0, k < L.nz - 1};
        const int off[6] = {-1, 1, -L.nx, L.nx, -L.nx * L.ny, L.nx * L.ny};
        const double coef[6] = {L.ax, L.ax, L.ay, L.ay, L.az, L.az};
        for (int q = 0; q < 6; ++q)
            if (has[q]) {
                M[(size_t)r * n + r + off[q]] += coef[q];
                M[(size_t)r * n + r] -= coef[q];
            }
    }
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int r = col + 1; r < n; ++r)
            if (fabs(M[(size_t)r * n + col]) > fabs(M[(size_t)piv * n + col])) piv = r;
        if (M[(size_t)piv * n + col] == 0.0) return false;
        if (piv != col)
            for (int q = 0; q < n; ++q) {
                std::swap(M[(size_t)piv * n + q], M[(size_t)col * n + q]);
                std::swap(inv[(size_t)piv * n + q], inv[(size_t)col * n + q]);
            }
        const double d = 1.0 / M[(size_t)col * n + col];
        for (int q = 0; q < n; ++q) {
            M[(size_t)col * n + q] *= d;
            inv[(size_t)col * n + q] *= d;
        }
        for (int r = 0; r < n; ++r) {
            if (r == col) continue;
            const double f = M[(size_t)r * n + col];
            if (f == 0.0) continue;
            for (int q = 0; q < n; ++q) {
                M[(size_t)r * n + q] -= f * M[(size_t)col * n + q];
                inv[(size_t)r * n + q] -= f * inv[(size_t)col * n + q];
            }
        }
    }
    return true;
}

cudaError_t mg_create(const Geom& g, int mode, MgSolver* m, cudaStream_t s, size_t* bytes, int* alloc_no,
                      int fail_at) {
    *m = MgSolver{};
    m->mode = mode;
    m->pairs = 1;
    if (const char* v = getenv("VOF_MG_PAIRS")) m->pairs = atoi(v) != 0;
    m->nlev = mg_plan(g, m->lv, MG_MAX_LEVELS);
    cudaError_t e;
    const size_t vb = mode == MG_MIXED ? sizeof(__nv_bfloat16) : sizeof(double);
    const size_t cb = mode == MG_MIXED ? sizeof(float) : sizeof(double);
    const MgLevel& Lc = m->lv[m->nlev - 1];
    // The tail: the deepest run of levels (at most MG_TAIL_CELLS cells each)
    // whose vectors and dense coarse inverse fit in MG_TAIL_SMEM bytes.
    const bool dense_ok = Lc.ncell <= MG_DENSE_MAX;
    const size_t inv_bytes = dense_ok ? (size_t)Lc.ncell * Lc.ncell * cb : 0;
    m->tail = m->nlev;
    m->tail_smem = 0;
    {
        size_t acc = inv_bytes;
        for (int l = m->nlev - 1; l >= 0; --l) {
            const size_t lb = 3 * (size_t)tail_vec_bytes(m->lv[l].ncell, (int)vb);
            if (m->lv[l].ncell > MG_TAIL_CELLS || acc + lb > MG_TAIL_SMEM) break;
            acc += lb;
            m->tail = l;
            m->tail_smem = (int)acc;
        }
    }
    m->dense = (m->tail < m->nlev) && dense_ok;
    if (m->tail < m->nlev) {
        e = mode == MG_MIXED ? cudaFuncSetAttribute(k_mg_tail<__nv_bfloat16>,
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize, m->tail_smem)
                             : cudaFuncSetAttribute(k_mg_tail<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    m->tail_smem);
        if (e != cudaSuccess) return e;
    }
    auto alloc = [&](void** p, size_t nb) -> cudaError_t {
        if (alloc_no && (*alloc_no)++ == fail_at) {  // injected (vof_debug_fail_alloc)
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
        cudaError_t r = cudaMalloc(p, nb);
        if (r != cudaSuccess) {
            *p = nullptr;
            return r;
        }
        *bytes += nb;
        return cudaMemsetAsync(*p, 0, nb, s);
    };
    int maxblk = 1;
    for (int l = 0; l < m->nlev; ++l) {
        MgLevel& L = m->lv[l];
        const size_t nb = (size_t)L.ncell * vb;
        if ((e = alloc(&L.e0, nb)) != cudaSuccess || (e = alloc(&L.e1, nb)) != cudaSuccess ||
            (e = alloc(&L.b, nb)) != cudaSuccess)
            return e;
        const int blk = L.gx * L.gy * L.gz;
        maxblk = blk > maxblk ? blk : maxblk;
    }
    m->nblk = m->lv[0].gx * m->lv[0].gy * m->lv[0].gz;
    if ((e = alloc((void**)&m->d_partial, sizeof(double) * 2 * maxblk)) != cudaSuccess ||
        (e = alloc((void**)&m->d_result, sizeof(double) * 8)) != cudaSuccess ||
        (e = alloc((void**)&m->d_lv, sizeof(MgLevel) * m->nlev)) != cudaSuccess)
        return e;
    if ((e = cudaHostAlloc((void**)&m->h_result, sizeof(double) * 2, cudaHostAllocMapped)) != cudaSuccess) {
        m->h_result = nullptr;
        return e;
    }
    if ((e = cudaHostGetDevicePointer((void**)&m->h_result_dev, m->h_result, 0)) != cudaSuccess) return e;
    if (m->dense) {
        std::vector<double> inv;
        if (!dense_inverse(Lc, inv)) return cudaErrorInvalidValue;
        if ((e = alloc(&m->d_cinv, inv.size() * cb)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        if (mode == MG_MIXED) {
            std::vector<float> f(inv.begin(), inv.end());
            e = cudaMemcpy(m->d_cinv, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice);
        } else {
            e = cudaMemcpy(m->d_cinv, inv.data(), inv.size() * sizeof(double), cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) return e;
    }
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    return cudaMemcpy(m->d_lv, m->lv, sizeof(MgLevel) * m->nlev, cudaMemcpyHostToDevice);
}

void mg_destroy(MgSolver* m) {
    for (int l = 0; l < m->nlev; ++l) {
        if (m->lv[l].e0) cudaFree(m->lv[l].e0);
        if (m->lv[l].e1) cudaFree(m->lv[l].e1);
        if (m->lv[l].b) cudaFree(m->lv[l].b);
    }
    if (m->d_lv) cudaFree(m->d_lv);
    if (m->d_cinv) cudaFree(m->d_cinv);
    if (m->d_partial) cudaFree(m->d_partial);
    if (m->d_result) cudaFree(m->d_result);
    if (m->h_result) cudaFreeHost(m->h_result);
    if (m->iter_graph) cudaGraphExecDestroy(m->iter_graph);
    *m = MgSolver{};
}

static dim3 grid_of(const MgLevel& L) { return dim3(L.gx, L.gy, L.gz); }
static const dim3 kBlock(MG_BX, MG_BY, 1);

// Which buffer holds the final correction of level l after a V-cycle: a
// smoothed level ends on e1 (first step into e0, then nu - 1 + nu more);
// the coarsest on e0 (dense) or after MG_COARSE_SWEEPS sweeps.
static void* final_buffer(const MgSolver& m, int l) {
    const MgLevel& L = m.lv[l];
    if (l == m.nlev - 1) return (m.dense || !((MG_COARSE_SWEEPS - 1) & 1)) ? L.e0 : L.e1;
    return L.e1;
}

// One smoothing step of a multi-block level: on BF16 levels of even width
// the flat paired kernel (or, with m.pairs = 0, the row-paired one), the
// generic one otherwise.
template <typename S>
static void smooth(const MgSolver& m, const MgLevel& L, const S* ein, S* eout, const S* b, double ca, double cb,
                   bool read_prev, cudaStream_t s) {
    if constexpr (sizeof(S) == 2) {
        if ((L.nx & 1) == 0 && m.pairs) {
            const dim3 gp(L.pgx, L.pgz);
            const unsigned* wi = reinterpret_cast<const unsigned*>(ein);
            unsigned* wo = reinterpret_cast<unsigned*>(eout);
            const unsigned* wb = reinterpret_cast<const unsigned*>(b);
            if (read_prev)
                pdl_launch(k_mg_smooth_pairs<true>, gp, MG_FLAT_THREADS, 0, s, L, wi, wo, wb, (float)ca, (float)cb);
            else
                pdl_launch(k_mg_smooth_pairs<false>, gp, MG_FLAT_THREADS, 0, s, L, wi, wo, wb, (float)ca, (float)cb);
            return;
        }
        if ((L.nx & 1) == 0) {
            const dim3 g2((L.nx / 2 + MG_BX - 1) / MG_BX, L.gy, L.gz);
            pdl_launch(k_mg_smooth2, g2, kBlock, 0, s, L, ein, eout, b, ca, cb, read_prev ? 1 : 0);
            return;
        }
    }
    pdl_launch(k_mg_smooth<S>, grid_of(L), kBlock, 0, s, L, ein, eout, b, nullptr, ca, cb, read_prev);
}

// A level above the one-block tail that is smoothed by multi-block kernels.
static bool multi(const MgSolver& m, int l) { return l < m.tail && l < m.nlev - 1; }

// Restriction from / prolongation to level L by the flat paired kernels
// (BF16 vectors, 2 x 2 x 2 coarsening).
static bool pairs2(const MgSolver& m, const MgLevel& L) {
    return m.pairs && m.mode == MG_MIXED && L.rx == 2 && L.ry == 2 && L.rz == 2;
}

template <typename S>
static cudaError_t vcycle(const Geom& g, MgSolver& m, double* p64, cudaStream_t s, int& launches) {
    using C = typename St<S>::C;
    int pre_cur[MG_MAX_LEVELS] = {};
    int l = 0;
    for (; multi(m, l); ++l) {
        const MgLevel& L = m.lv[l];
        S* e[2] = {static_cast<S*>(L.e0), static_cast<S*>(L.e1)};
        const S* b = static_cast<const S*>(L.b);
        int cur = 0;  // the first step (from zero) was written together with b
        for (int q = 1; q < L.nu; ++q, cur ^= 1, ++launches)
            smooth<S>(m, L, e[cur], e[cur ^ 1], b, L.ca[q], L.cb[q], q >= 2, s);
        const MgLevel& Cl = m.lv[l + 1];
        S* ec = multi(m, l + 1) ? static_cast<S*>(Cl.e0) : nullptr;
        if (sizeof(S) == 2 && pairs2(m, L))
            pdl_launch(k_mg_restrict_pairs, dim3(Cl.cgx, Cl.cgz), MG_FLAT_THREADS, 0, s, L,
                       reinterpret_cast<const unsigned*>(e[cur]), reinterpret_cast<const unsigned*>(b), Cl,
                       reinterpret_cast<__nv_bfloat16*>(Cl.b), reinterpret_cast<__nv_bfloat16*>(ec));
        else if (L.rx * L.ry * L.rz > 8)
            pdl_launch(k_mg_restrict_wide<S>, Cl.ncell, RW_THREADS, 0, s, L, e[cur], b, Cl, static_cast<S*>(Cl.b),
                       ec);
        else
            pdl_launch(k_mg_restrict<S>, grid_of(Cl), kBlock, 0, s, L, e[cur], b, Cl, static_cast<S*>(Cl.b), ec);
        ++launches;
        pre_cur[l] = cur;
    }
    if (m.tail < m.nlev) {
        pdl_launch(k_mg_tail<S>, 1, TAIL_THREADS, m.tail_smem, s, m.d_lv + m.tail, m.nlev - m.tail,
                   static_cast<const C*>(m.d_cinv), static_cast<S*>(final_buffer(m, m.tail)));
        ++launches;
    } else {  // large coarsest level below no tail: mean-free sweeps from zero
        const MgLevel& L = m.lv[l];
        S* e[2] = {static_cast<S*>(L.e0), static_cast<S*>(L.e1)};
        const S* b = static_cast<const S*>(L.b);
        pdl_launch(k_level_sum<S>, grid_of(L), kBlock, 0, s, L, b, m.d_partial);
        pdl_launch(k_fold2, 1, MG_THREADS, 0, s, m.d_partial, L.gx * L.gy * L.gz, m.d_result + 6, nullptr);
        pdl_launch(k_mg_smooth<S>, grid_of(L), kBlock, 0, s, L, nullptr, e[0], b, m.d_result + 6, 0.0, MG_OMEGA,
                   0);
        launches += 3;
        for (int q = 1; q < MG_COARSE_SWEEPS; ++q, ++launches)
            pdl_launch(k_mg_smooth<S>, grid_of(L), kBlock, 0, s, L, e[(q - 1) & 1], e[q & 1], b, m.d_result + 6,
                       0.0, MG_OMEGA, 0);
    }
    for (int lc = l - 1; lc >= 0; --lc) {
        const MgLevel& L = m.lv[lc];
        const MgLevel& Cl = m.lv[lc + 1];
        S* e[2] = {static_cast<S*>(L.e0), static_cast<S*>(L.e1)};
        const S* b = static_cast<const S*>(L.b);
        int cur = pre_cur[lc];
        if (sizeof(S) == 2 && pairs2(m, L))
            pdl_launch(k_mg_prolong_pairs, dim3(Cl.cgx, Cl.cgz), MG_FLAT_THREADS, 0, s, L,
                       reinterpret_cast<unsigned*>(e[cur]), Cl,
                       static_cast<const __nv_bfloat16*>(final_buffer(m, lc + 1)));
        else
            pdl_launch(k_mg_prolong<S>, grid_of(L), kBlock, 0, s, L, e[cur], Cl,
                       static_cast<const S*>(final_buffer(m, lc + 1)));
        ++launches;
        for (int q = 0; q < L.nu; ++q, cur ^= 1, ++launches) {
            if (lc == 0 && q == L.nu - 1)
                pdl_launch(k_smooth_update<S>, grid_of(L), kBlock, 0, s, g, L, e[cur], e[cur ^ 1], b, p64, L.ca[q],
                           L.cb[q], q >= 1);
            else
                smooth<S>(m, L, e[cur], e[cur ^ 1], b, L.ca[q], L.cb[q], q >= 1, s);
        }
    }
    if (l == 0) {  // the fine level was solved by the tail or as the coarsest level
        pdl_launch(k_update64<S>, grid_of(m.lv[0]), kBlock, 0, s, g, m.lv[0], p64,
                   static_cast<const S*>(final_buffer(m, 0)));
        ++launches;
    }
    return cudaGetLastError();
}

cudaError_t mg_widen(const Geom& g, const MgSolver& m, const float* p32, double* p64, cudaStream_t s) {
    pdl_launch(k_widen, grid_of(m.lv[0]), kBlock, 0, s, g, m.lv[0], p32, p64);
    return cudaGetLastError();
}

// One outer iteration after the first residual: V-cycle with p += e, then the
// new residual and its norm (also written to the mapped host copy).
template <typename S, typename R>
static cudaError_t outer_iteration(const Geom& g, MgSolver& m, const R* rhs, double* p64, cudaStream_t s,
                                   int& launches) {
    cudaError_t e = vcycle<S>(g, m, p64, s, launches);
    if (e != cudaSuccess) return e;
    const MgLevel& L0 = m.lv[0];
    pdl_launch(k_resid0<S, R>, grid_of(L0), kBlock, 0, s, g, L0, rhs, m.d_result + 2, p64, static_cast<S*>(L0.b),
               multi(m, 0) ? static_cast<S*>(L0.e0) : nullptr, m.d_partial);
    pdl_launch(k_fold2, 1, MG_THREADS, 0, s, m.d_partial, m.nblk, m.d_result, m.h_result_dev);
    launches += 2;
    return cudaGetLastError();
}

template <typename S, typename R>
static cudaError_t capture_iteration(const Geom& g, MgSolver& m, const R* rhs, double* p64, float* p32,
                                     cudaStream_t cap) {
    if (m.iter_graph) {
        cudaGraphExecDestroy(m.iter_graph);
        m.iter_graph = nullptr;
    }
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    int launches = 0;
    const cudaError_t e1 = outer_iteration<S, R>(g, m, rhs, p64, cap, launches);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(cap, &graph);
    if (e1 != cudaSuccess || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return e1 != cudaSuccess ? e1 : e;
    }
    e = cudaGraphInstantiate(&m.iter_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        m.iter_graph = nullptr;
        return e;
    }
    m.graph_key[0] = rhs;
    m.graph_key[1] = p64;
    m.graph_key[2] = p32;
    m.graph_launches = launches;
    return cudaSuccess;
}

template <typename S, typename R>
static cudaError_t solve_impl(const Geom& g, MgSolver& m, const R* rhs, double* p64, float* p32, double tol,
                              int max_outer, MgStats* st, cudaStream_t s, cudaStream_t cap) {
    const MgLevel& L0 = m.lv[0];
    const dim3 grid = grid_of(L0);
    double* part = m.d_partial;
    double* res = m.d_result;
    cudaError_t e;
    if (!m.iter_graph || m.graph_key[0] != rhs || m.graph_key[1] != p64 || m.graph_key[2] != p32)
        if ((e = capture_iteration<S, R>(g, m, rhs, p64, p32, cap)) != cudaSuccess) return e;
    int launches = 0;
    pdl_launch(k_sum_rhs<R>, grid, kBlock, 0, s, g, L0, rhs, part);
    pdl_launch(k_fold2, 1, MG_THREADS, 0, s, part, m.nblk, res + 2, nullptr);
    pdl_launch(k_resid0<S, R>, grid, kBlock, 0, s, g, L0, rhs, res + 2, p64, static_cast<S*>(L0.b),
               multi(m, 0) ? static_cast<S*>(L0.e0) : nullptr, part);
    pdl_launch(k_fold2, 1, MG_THREADS, 0, s, part, m.nblk, res, m.h_result_dev);
    launches += 4;
    int it = 0;
    double rel = 0, r0 = -1;
    for (;; ++it) {
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        const double rr = m.h_result[0], bb = m.h_result[1];
        rel = bb > 0 ? sqrt(rr / bb) : 0.0;
        if (r0 < 0) r0 = rel;
        if (rel <= tol || it >= max_outer) break;
        if ((e = cudaGraphLaunch(m.iter_graph, s)) != cudaSuccess) return e;
        launches += m.graph_launches;
    }
    pdl_launch(k_sum_p, grid, kBlock, 0, s, g, L0, p64, part);
    pdl_launch(k_fold2, 1, MG_THREADS, 0, s, part, m.nblk, res + 4, nullptr);
    pdl_launch(k_gauge_cast, grid, kBlock, 0, s, g, L0, p64, res + 4, p32);
    launches += 3;
    if (st) {
        st->outer = it;
        st->rel_initial = r0;
        st->rel_final = rel;
        st->launches = launches;
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return rel <= tol ? cudaSuccess : cudaErrorNotReady;
}

cudaError_t mg_solve(const Geom& g, MgSolver& m, const float* rhs, double* p64, float* p32, double tol,
                     int max_outer, MgStats* st, cudaStream_t s, cudaStream_t cap) {
    if (m.mode == MG_MIXED)
        return solve_impl<__nv_bfloat16, float>(g, m, rhs, p64, p32, tol, max_outer, st, s, cap);
    return solve_impl<double, float>(g, m, rhs, p64, p32, tol, max_outer, st, s, cap);
}

cudaError_t mg_solve64(const Geom& g, MgSolver& m, const double* rhs, double* p64, double tol, int max_outer,
                       MgStats* st, cudaStream_t s, cudaStream_t cap) {
    if (m.mode == MG_MIXED)
        return solve_impl<__nv_bfloat16, double>(g, m, rhs, p64, nullptr, tol, max_outer, st, s, cap);
    return solve_impl<double, double>(g, m, rhs, p64, nullptr, tol, max_outer, st, s, cap);
}

}  // namespace vof
