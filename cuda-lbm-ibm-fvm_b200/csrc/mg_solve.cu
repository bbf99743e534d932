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
// V-cycle: damped Jacobi (omega = 6/7, the Jacobi update of the reference's
// sweep with damping) as the smoother, 2 pre + 2 post sweeps on large levels
// and 8 + 8 on levels no wider than 25 cells, averaging restriction,
// cell-centred multilinear prolongation with zero-gradient ends, coarse
// operators rediscretised at the coarse spacing.  Each axis is coarsened by
// its smallest prime factor (2, 3, 5, 7) while at least two cells remain
// (200 -> 100 -> 50 -> 25 -> 5); the coarsest level gets 100 Jacobi sweeps
// after removing its mean.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>

#include "mg_solve.h"

namespace vof {

template <typename S>
struct St;
template <>
struct St<__nv_bfloat16> {
    using C = float;
    __device__ static float ld(const __nv_bfloat16* p, long i) { return __bfloat162float(p[i]); }
    __device__ static void st(__nv_bfloat16* p, long i, float v) { p[i] = __float2bfloat16_rn(v); }
};
template <>
struct St<double> {
    using C = double;
    __device__ static double ld(const double* p, long i) { return p[i]; }
    __device__ static void st(double* p, long i, double v) { p[i] = v; }
};

constexpr int MG_THREADS = 256;
constexpr int MG_RED_BLOCKS = 296;

__device__ __forceinline__ long lidx(const MgLevel& L, int i, int j, int k) {
    return ((long)k * L.ny + j) * L.nx + i;
}

// (A e)_c and the diagonal of A at (i,j,k) of level L.
template <typename S, typename C>
__device__ __forceinline__ void apply_row(const MgLevel& L, const S* e, int i, int j, int k, C& Ae, C& dg) {
    using T = St<S>;
    const long c = lidx(L, i, j, k);
    const C ec = T::ld(e, c);
    const C ax = (C)L.ax, ay = (C)L.ay, az = (C)L.az;
    C s = 0, d = 0;
    if (i > 0) { s += ax * ((C)T::ld(e, c - 1) - ec); d -= ax; }
    if (i < L.nx - 1) { s += ax * ((C)T::ld(e, c + 1) - ec); d -= ax; }
    if (j > 0) { s += ay * ((C)T::ld(e, c - L.nx) - ec); d -= ay; }
    if (j < L.ny - 1) { s += ay * ((C)T::ld(e, c + L.nx) - ec); d -= ay; }
    if (k > 0) { s += az * ((C)T::ld(e, c - (long)L.nx * L.ny) - ec); d -= az; }
    if (k < L.nz - 1) { s += az * ((C)T::ld(e, c + (long)L.nx * L.ny) - ec); d -= az; }
    Ae = s;
    dg = d;
}

#define MG_FOR_CELLS(L, i, j, k)                                                                   \
    for (long t_ = (long)blockIdx.x * blockDim.x + threadIdx.x, n_ = (long)(L).nx * (L).ny * (L).nz; \
         t_ < n_; t_ += (long)gridDim.x * blockDim.x)                                              \
        for (int i = (int)(t_ % (L).nx), j = (int)((t_ / (L).nx) % (L).ny),                       \
                 k = (int)(t_ / ((long)(L).nx * (L).ny)), once_ = 1;                               \
             once_; once_ = 0)

// Damped Jacobi sweep: eout = ein + w (b - A ein) / diag (ein == nullptr: ein = 0).
template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_mg_jacobi(MgLevel L, const S* __restrict__ ein,
                                                          S* __restrict__ eout, const S* __restrict__ b,
                                                          double omega) {
    using T = St<S>;
    using C = typename T::C;
    MG_FOR_CELLS(L, i, j, k) {
        const long c = lidx(L, i, j, k);
        C Ae = 0, dg = 0;
        if (ein) {
            apply_row<S, C>(L, ein, i, j, k, Ae, dg);
        } else {
            const C ax = (C)L.ax, ay = (C)L.ay, az = (C)L.az;
            dg = -(ax * ((i > 0) + (i < L.nx - 1)) + ay * ((j > 0) + (j < L.ny - 1)) + az * ((k > 0) + (k < L.nz - 1)));
        }
        const C e0 = ein ? (C)T::ld(ein, c) : (C)0;
        const C r = (C)T::ld(b, c) - Ae;
        T::st(eout, c, dg != 0 ? e0 + (C)omega * r / dg : e0);
    }
}

// bc = average over the fine cells of each coarse cell of (b - A e).
template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_mg_restrict(MgLevel F, const S* __restrict__ e,
                                                            const S* __restrict__ b, MgLevel Cl,
                                                            S* __restrict__ bc) {
    using T = St<S>;
    using C = typename T::C;
    MG_FOR_CELLS(Cl, I, J, K) {
        C acc = 0;
        for (int dk = 0; dk < F.rz; ++dk)
            for (int dj = 0; dj < F.ry; ++dj)
                for (int di = 0; di < F.rx; ++di) {
                    const int i = I * F.rx + di, j = J * F.ry + dj, k = K * F.rz + dk;
                    C Ae, dg;
                    apply_row<S, C>(F, e, i, j, k, Ae, dg);
                    acc += (C)T::ld(b, lidx(F, i, j, k)) - Ae;
                }
        T::st(bc, lidx(Cl, I, J, K), acc / (C)(F.rx * F.ry * F.rz));
    }
}

// Cell-centred linear interpolation weight along one axis: fine cell x of a
// level coarsened by r; returns the two coarse indices and the weight of hi.
template <typename C>
__device__ __forceinline__ void lin1(int x, int r, int nc, int& lo, int& hi, C& t) {
    if (r == 1) {
        lo = hi = x;
        t = 0;
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

// e += P ec (multilinear, zero-gradient beyond the coarse ends).
template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_mg_prolong(MgLevel F, S* __restrict__ e, MgLevel Cl,
                                                           const S* __restrict__ ec) {
    using T = St<S>;
    using C = typename T::C;
    MG_FOR_CELLS(F, i, j, k) {
        int x0, x1, y0, y1, z0, z1;
        C tx, ty, tz;
        lin1<C>(i, F.rx, Cl.nx, x0, x1, tx);
        lin1<C>(j, F.ry, Cl.ny, y0, y1, ty);
        lin1<C>(k, F.rz, Cl.nz, z0, z1, tz);
        auto at = [&](int a, int bb, int cc) { return (C)T::ld(ec, lidx(Cl, a, bb, cc)); };
        const C c00 = at(x0, y0, z0) * (1 - tx) + at(x1, y0, z0) * tx;
        const C c10 = at(x0, y1, z0) * (1 - tx) + at(x1, y1, z0) * tx;
        const C c01 = at(x0, y0, z1) * (1 - tx) + at(x1, y0, z1) * tx;
        const C c11 = at(x0, y1, z1) * (1 - tx) + at(x1, y1, z1) * tx;
        const C v = (c00 * (1 - ty) + c10 * ty) * (1 - tz) + (c01 * (1 - ty) + c11 * ty) * tz;
        const long c = lidx(F, i, j, k);
        T::st(e, c, (C)T::ld(e, c) + v);
    }
}

// Coarsest level, one block: remove the mean of b, then `sweeps` damped
// Jacobi sweeps from e = 0 in shared memory.
template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_mg_coarsest(MgLevel L, const S* __restrict__ b, S* __restrict__ e,
                                                            int sweeps, double omega) {
    using T = St<S>;
    using C = typename T::C;
    extern __shared__ __align__(16) unsigned char raw[];
    C* sb = reinterpret_cast<C*>(raw);
    C* s0 = sb + L.ncell;
    C* s1 = s0 + L.ncell;
    __shared__ double red[MG_THREADS];
    double acc = 0;
    for (int c = threadIdx.x; c < L.ncell; c += MG_THREADS) {
        sb[c] = (C)T::ld(b, c);
        s0[c] = 0;
        acc += (double)sb[c];
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int q = 0; q < MG_THREADS; ++q) s += red[q];
        red[0] = s / L.ncell;
    }
    __syncthreads();
    const C mean = (C)red[0];
    for (int c = threadIdx.x; c < L.ncell; c += MG_THREADS) sb[c] -= mean;
    __syncthreads();
    const C ax = (C)L.ax, ay = (C)L.ay, az = (C)L.az;
    for (int sw = 0; sw < sweeps; ++sw) {
        const C* in = (sw & 1) ? s1 : s0;
        C* out = (sw & 1) ? s0 : s1;
        for (int c = threadIdx.x; c < L.ncell; c += MG_THREADS) {
            const int i = c % L.nx, j = (c / L.nx) % L.ny, k = c / (L.nx * L.ny);
            const C ev = in[c];
            C s = 0, d = 0;
            if (i > 0) { s += ax * (in[c - 1] - ev); d -= ax; }
            if (i < L.nx - 1) { s += ax * (in[c + 1] - ev); d -= ax; }
            if (j > 0) { s += ay * (in[c - L.nx] - ev); d -= ay; }
            if (j < L.ny - 1) { s += ay * (in[c + L.nx] - ev); d -= ay; }
            if (k > 0) { s += az * (in[c - L.nx * L.ny] - ev); d -= az; }
            if (k < L.nz - 1) { s += az * (in[c + L.nx * L.ny] - ev); d -= az; }
            out[c] = d != 0 ? ev + (C)omega * (sb[c] - s) / d : ev;
        }
        __syncthreads();
    }
    const C* fin = (sweeps & 1) ? s1 : s0;
    for (int c = threadIdx.x; c < L.ncell; c += MG_THREADS) T::st(e, c, fin[c]);
}

// ---- fine level, FP64 -------------------------------------------------------
// Deterministic block reduction of up to 2 doubles into partial[2*block + v].
__device__ void block_sum2(double a, double b, double* partial) {
    __shared__ double sh[2][MG_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][wid] = a;
        sh[1][wid] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0, y = 0;
        for (int q = 0; q < MG_THREADS / 32; ++q) {
            x += sh[0][q];
            y += sh[1][q];
        }
        partial[2 * blockIdx.x] = x;
        partial[2 * blockIdx.x + 1] = y;
    }
}

__global__ void __launch_bounds__(MG_THREADS) k_fold2(const double* partial, int nblk, double* out) {
    __shared__ double sh[2][MG_THREADS];
    double a = 0, b = 0;
    for (int q = threadIdx.x; q < nblk; q += MG_THREADS) {
        a += partial[2 * q];
        b += partial[2 * q + 1];
    }
    sh[0][threadIdx.x] = a;
    sh[1][threadIdx.x] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0, y = 0;
        for (int q = 0; q < MG_THREADS; ++q) {
            x += sh[0][q];
            y += sh[1][q];
        }
        out[0] = x;
        out[1] = y;
    }
}

#define FINE_FOR(g, i, j, k)                                                                   \
    for (long t_ = (long)blockIdx.x * blockDim.x + threadIdx.x, n_ = (long)(g).nx * (g).ny * (g).nz; \
         t_ < n_; t_ += (long)gridDim.x * blockDim.x)                                          \
        for (int i = 1 + (int)(t_ % (g).nx), j = 1 + (int)((t_ / (g).nx) % (g).ny),           \
                 k = 1 + (int)(t_ / ((long)(g).nx * (g).ny)), once_ = 1;                       \
             once_; once_ = 0)

// Sum of rhs over the interior (for its mean).
__global__ void __launch_bounds__(MG_THREADS) k_sum_rhs(Geom g, const float* __restrict__ rhs, double* partial) {
    double a = 0;
    FINE_FOR(g, i, j, k) a += (double)rhs[gidx(g, i, j, k)];
    block_sum2(a, 0.0, partial);
}

// r = (rhs - mean) - A p64 in FP64; r stored in the inner precision at the
// fine multigrid level; partial sums of r^2 and b^2.
template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_residual64(Geom g, const float* __restrict__ rhs,
                                                           const double* __restrict__ meanp,
                                                           const double* __restrict__ p, S* __restrict__ r_out,
                                                           double* partial) {
    using T = St<S>;
    const double mean = meanp[0] / ((double)g.nx * g.ny * g.nz);
    const double ax = (double)g.dxi * g.dxi, ay = (double)g.dyi * g.dyi, az = (double)g.dzi * g.dzi;
    double rr = 0, bb = 0;
    FINE_FOR(g, i, j, k) {
        const int id = gidx(g, i, j, k);
        const double pc = p[id];
        double s = 0;
        if (i > 1) s += ax * (p[id - 1] - pc);
        if (i < g.nx) s += ax * (p[id + 1] - pc);
        if (j > 1) s += ay * (p[id - g.px] - pc);
        if (j < g.ny) s += ay * (p[id + g.px] - pc);
        if (k > 1) s += az * (p[id - g.plane] - pc);
        if (k < g.nz) s += az * (p[id + g.plane] - pc);
        const double b = (double)rhs[id] - mean;
        const double r = b - s;
        rr += r * r;
        bb += b * b;
        T::st(r_out, ((long)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1), (typename T::C)r);
    }
    block_sum2(rr, bb, partial);
}

// p64 += e (the inner correction, widened to FP64).
template <typename S>
__global__ void __launch_bounds__(MG_THREADS) k_update64(Geom g, double* __restrict__ p, const S* __restrict__ e) {
    using T = St<S>;
    FINE_FOR(g, i, j, k) {
        const int id = gidx(g, i, j, k);
        p[id] += (double)T::ld(e, ((long)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1));
    }
}

// Sum of p64 over the interior (for the gauge).
__global__ void __launch_bounds__(MG_THREADS) k_sum_p(Geom g, const double* __restrict__ p, double* partial) {
    double a = 0;
    FINE_FOR(g, i, j, k) a += p[gidx(g, i, j, k)];
    block_sum2(a, 0.0, partial);
}

// p64 -= mean (gauge mean(p) = 0); p32 = float(p64) on the interior.
__global__ void __launch_bounds__(MG_THREADS) k_gauge_cast(Geom g, double* __restrict__ p,
                                                           const double* __restrict__ sump, float* __restrict__ p32) {
    const double mean = sump[0] / ((double)g.nx * g.ny * g.nz);
    FINE_FOR(g, i, j, k) {
        const int id = gidx(g, i, j, k);
        const double v = p[id] - mean;
        p[id] = v;
        p32[id] = (float)v;
    }
}

// p64 = double(p32) on the interior (after an upload of P).
__global__ void __launch_bounds__(MG_THREADS) k_widen(Geom g, const float* __restrict__ p32, double* __restrict__ p) {
    FINE_FOR(g, i, j, k) {
        const int id = gidx(g, i, j, k);
        p[id] = (double)p32[id];
    }
}

// ---- host -------------------------------------------------------------------
static int smallest_factor(int n) {
    const int f[4] = {2, 3, 5, 7};
    for (int q = 0; q < 4; ++q)
        if (n % f[q] == 0 && n / f[q] >= 2) return f[q];
    return 1;
}

int mg_plan(const Geom& g, MgLevel* lv, int max_levels) {
    int n[3] = {g.nx, g.ny, g.nz};
    double h[3] = {(double)g.dx, (double)g.dy, (double)g.dz};
    int L = 0;
    while (L < max_levels) {
        MgLevel& m = lv[L];
        m.nx = n[0];
        m.ny = n[1];
        m.nz = n[2];
        m.ncell = n[0] * n[1] * n[2];
        m.ax = 1.0 / (h[0] * h[0]);
        m.ay = 1.0 / (h[1] * h[1]);
        m.az = 1.0 / (h[2] * h[2]);
        int r[3];
        for (int a = 0; a < 3; ++a) r[a] = (n[a] > 2) ? smallest_factor(n[a]) : 1;
        const bool last = (r[0] == 1 && r[1] == 1 && r[2] == 1) || (n[0] <= 3 && n[1] <= 3 && n[2] <= 3) ||
                          L == max_levels - 1;
        m.rx = last ? 1 : r[0];
        m.ry = last ? 1 : r[1];
        m.rz = last ? 1 : r[2];
        ++L;
        if (last) break;
        for (int a = 0; a < 3; ++a) {
            n[a] /= r[a];
            h[a] *= r[a];
        }
    }
    return L;
}

size_t mg_storage_bytes(int mode) { return mode == MG_MIXED ? 2 : 8; }

// Kernel launches of one V-cycle from level l down (for the launch count).
static int vcycle_launches(const MgSolver& m, int l) {
    const MgLevel& L = m.lv[l];
    if (l == m.nlev - 1) {
        const size_t smem = 3 * (size_t)L.ncell * (m.mode == MG_MIXED ? sizeof(float) : sizeof(double));
        return smem <= 200 * 1024 ? 1 : MG_COARSE_SWEEPS;
    }
    const int nu = (L.nx > 25 || L.ny > 25 || L.nz > 25) ? MG_NU_FINE : MG_NU_COARSE;
    return 2 * nu + 2 + vcycle_launches(m, l + 1);
}

template <typename S>
static cudaError_t vcycle(MgSolver& m, int l, cudaStream_t s) {
    MgLevel& L = m.lv[l];
    S* b = static_cast<S*>(L.b);
    S* e[2] = {static_cast<S*>(L.e0), static_cast<S*>(L.e1)};
    const int blocks = (int)((L.ncell + MG_THREADS - 1) / MG_THREADS) < 148 * 8
                           ? (int)((L.ncell + MG_THREADS - 1) / MG_THREADS) : 148 * 8;
    if (l == m.nlev - 1) {
        const size_t smem = 3 * (size_t)L.ncell * sizeof(typename St<S>::C);
        if (smem <= 200 * 1024) {
            k_mg_coarsest<S><<<1, MG_THREADS, smem, s>>>(L, b, e[0], MG_COARSE_SWEEPS, MG_OMEGA);
            L.cur = 0;
            return cudaGetLastError();
        }
        // large coarsest level: plain sweeps
        k_mg_jacobi<S><<<blocks, MG_THREADS, 0, s>>>(L, nullptr, e[0], b, MG_OMEGA);
        for (int q = 1; q < MG_COARSE_SWEEPS; ++q)
            k_mg_jacobi<S><<<blocks, MG_THREADS, 0, s>>>(L, e[(q - 1) & 1], e[q & 1], b, MG_OMEGA);
        L.cur = (MG_COARSE_SWEEPS - 1) & 1;
        return cudaGetLastError();
    }
    const int wide = L.nx > 25 || L.ny > 25 || L.nz > 25;
    const int nu = wide ? MG_NU_FINE : MG_NU_COARSE;
    int cur = 0;
    k_mg_jacobi<S><<<blocks, MG_THREADS, 0, s>>>(L, nullptr, e[0], b, MG_OMEGA);
    for (int q = 1; q < nu; ++q) {
        k_mg_jacobi<S><<<blocks, MG_THREADS, 0, s>>>(L, e[cur], e[cur ^ 1], b, MG_OMEGA);
        cur ^= 1;
    }
    MgLevel& Cl = m.lv[l + 1];
    const int cblocks = (int)((Cl.ncell + MG_THREADS - 1) / MG_THREADS) < 148 * 8
                            ? (int)((Cl.ncell + MG_THREADS - 1) / MG_THREADS) : 148 * 8;
    k_mg_restrict<S><<<cblocks, MG_THREADS, 0, s>>>(L, e[cur], b, Cl, static_cast<S*>(Cl.b));
    cudaError_t err = vcycle<S>(m, l + 1, s);
    if (err != cudaSuccess) return err;
    S* ec = static_cast<S*>(Cl.cur ? Cl.e1 : Cl.e0);
    k_mg_prolong<S><<<blocks, MG_THREADS, 0, s>>>(L, e[cur], Cl, ec);
    for (int q = 0; q < nu; ++q) {
        k_mg_jacobi<S><<<blocks, MG_THREADS, 0, s>>>(L, e[cur], e[cur ^ 1], b, MG_OMEGA);
        cur ^= 1;
    }
    L.cur = cur;
    return cudaGetLastError();
}

cudaError_t mg_configure(const MgSolver& m) {
    const MgLevel& L = m.lv[m.nlev - 1];
    const size_t smem = 3 * (size_t)L.ncell * (m.mode == MG_MIXED ? sizeof(float) : sizeof(double));
    if (smem > 200 * 1024) return cudaSuccess;
    return m.mode == MG_MIXED
               ? cudaFuncSetAttribute(k_mg_coarsest<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem)
               : cudaFuncSetAttribute(k_mg_coarsest<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

cudaError_t mg_widen(const Geom& g, const float* p32, double* p64, cudaStream_t s) {
    k_widen<<<148 * 8, MG_THREADS, 0, s>>>(g, p32, p64);
    return cudaGetLastError();
}

template <typename S>
static cudaError_t solve_impl(const Geom& g, MgSolver& m, const float* rhs, double* p64, float* p32,
                              double tol, int max_outer, MgStats* st, cudaStream_t s) {
    const int nblk = MG_RED_BLOCKS;
    double* part = m.d_partial;
    double* res = m.d_result;  // [0..1] fold of the residual, [2..3] sum of rhs, [4..5] sum of p
    cudaError_t e;
    k_sum_rhs<<<nblk, MG_THREADS, 0, s>>>(g, rhs, part);
    k_fold2<<<1, MG_THREADS, 0, s>>>(part, nblk, res + 2);
    int it = 0;
    double rel = 0, r0 = -1;
    for (;; ++it) {
        k_residual64<S><<<nblk, MG_THREADS, 0, s>>>(g, rhs, res + 2, p64, static_cast<S*>(m.lv[0].b), part);
        k_fold2<<<1, MG_THREADS, 0, s>>>(part, nblk, res);
        if ((e = cudaMemcpyAsync(m.h_result, res, 2 * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        const double rr = m.h_result[0], bb = m.h_result[1];
        rel = bb > 0 ? sqrt(rr / bb) : 0.0;
        if (r0 < 0) r0 = rel;
        if (rel <= tol || it >= max_outer) break;
        if ((e = vcycle<S>(m, 0, s)) != cudaSuccess) return e;
        const MgLevel& L0 = m.lv[0];
        k_update64<S><<<148 * 8, MG_THREADS, 0, s>>>(g, p64, static_cast<const S*>(L0.cur ? L0.e1 : L0.e0));
    }
    // gauge: mean(p) = 0, then the FP32 copy for the velocity correction
    k_sum_p<<<nblk, MG_THREADS, 0, s>>>(g, p64, part);
    k_fold2<<<1, MG_THREADS, 0, s>>>(part, nblk, res + 4);
    k_gauge_cast<<<148 * 8, MG_THREADS, 0, s>>>(g, p64, res + 4, p32);
    if (st) {
        st->outer = it;
        st->rel_initial = r0;
        st->rel_final = rel;
        st->launches = 2 + (it + 1) * 2 + it * (vcycle_launches(m, 0) + 1) + 3;
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return rel <= tol ? cudaSuccess : cudaErrorNotReady;
}

cudaError_t mg_solve(const Geom& g, MgSolver& m, const float* rhs, double* p64, float* p32, double tol,
                     int max_outer, MgStats* st, cudaStream_t s) {
    if (m.mode == MG_MIXED) return solve_impl<__nv_bfloat16>(g, m, rhs, p64, p32, tol, max_outer, st, s);
    return solve_impl<double>(g, m, rhs, p64, p32, tol, max_outer, st, s);
}

}  // namespace vof
