// jacobi_tb.cu -- Jacobi sweeps of the pressure system (solve_p_jacobi_kernel,
// voftrial1.cu:401-439, with the ping-pong of voftrial1.cu:1371-1375).  The
// default is one sweep per launch with two cells per thread and the plane
// cases peeled out of the z march (k_jacobi_peel), marching up or down.  The
// other kernels here, all with the same bits: the same without the peeling
// (k_jacobi_pairs), four cells per thread (k_jacobi_quad), own-column
// cp.async ring (k_jacobi_ring), rows fed by bulk copies (k_jacobi_bulk),
// one cell per thread (k_jacobi_col), two sweeps per launch
// (k_jacobi_pairs2), and T sweeps per launch temporally blocked in shared
// memory through TMA (k_jacobi_tb<T>, described below).
//
// Compiled with -fmad=false: each cell update keeps the reference's
//     pt = (rhs - ae*pE - aw*pW - an*pN - as*pS - af*pF - ab*pB) / ap
// with the same operand order, so T blocked sweeps give the same bits as T
// separate sweeps.  The division uses div_rn_pre with the IEEE reciprocal of
// ap (a handful of values per launch), which equals the IEEE quotient.
//
// Input planes (pressure and rhs) stream into a ring of shared-memory slots
// through TMA loads issued several planes ahead by one thread and completed
// on per-slot mbarriers, so HBM latency overlaps the sweeps of earlier planes.
//
// 2.5D pipeline.  A block owns BX x BY columns and walks a chunk of z planes.
// It keeps, for every level t < T, a ring of three planes of an extended tile
// (BX + 2T) x (BY + 2T) in shared memory.  When plane s of the input (level 0)
// arrives, level t is computed at plane s - t on the tile shrunk by T - t
// cells on each side, from level t-1 at planes s-t-1 .. s-t+1; level T, the
// tile interior, goes to global memory.  Ghost cells (and the never-written
// ghost planes) are carried unchanged from level to level: the reference
// never writes pressure ghosts, and they enter interior updates only through
// zero coefficients.
#include <cuda_runtime.h>
#include <stdlib.h>

#include "jacobi_tb.h"
#include "tma.cuh"

namespace vof {

#if defined(__CUDA_ARCH__) && !defined(VOF_FMAD_FALSE)
#error "jacobi_tb.cu must be compiled with -fmad=false -DVOF_FMAD_FALSE"
#endif

// Threads (32, 8).  The tile is BX = BY = 32 - 2(T-1) columns, so every
// level's rows (BX + 2(T-t) cells wide) fit one warp and each thread updates
// four rows per level and plane; the extended tile is always 34 x 34 cells.
constexpr int JB_TX = 32, JB_TY = 8, JB_THREADS = JB_TX * JB_TY, JB_ROWS = 4;
constexpr int JB_EX = JB_TX + 2, JB_EY = JB_TY * JB_ROWS + 2;
// TMA box: 40 x 34 x 1 floats from an x origin rounded down to a multiple of
// 4 elements (16 bytes); a plane slot is padded to a multiple of 128 bytes.
constexpr int JB_W = 40, JB_PLANE = JB_W * JB_EY, JB_PLANE_PAD = (JB_PLANE * 4 + 127) / 128 * 32;
constexpr uint32_t JB_BOX_BYTES = JB_PLANE * 4;

// Input planes in flight beyond those in use (the TMA prefetch depth).  One
// keeps the block at 49 KB of shared memory: four blocks (32 warps) per SM,
// which hides more latency than a deeper prefetch with three blocks (measured
// 5 % faster at 200^3).
#ifndef VOF_JB_AHEAD
#define VOF_JB_AHEAD 1
#endif
template <int T>
struct JTile {
    static constexpr int BX = JB_TX - 2 * (T - 1), BY = JB_TY * JB_ROWS - 2 * (T - 1);
    static constexpr int HOLD = T > 2 ? T : 2;  // steps a plane's slot stays in use
    static constexpr int SLOTS = HOLD + VOF_JB_AHEAD;
    static constexpr size_t SMEM = sizeof(float) * (size_t)(2 * SLOTS + 3 * (T - 1)) * JB_PLANE_PAD +
                                   sizeof(uint64_t) * SLOTS;
};

template <int T>
__global__ void __launch_bounds__(JB_THREADS) k_jacobi_tb(Geom g, const __grid_constant__ CUtensorMap map_p,
                                                         const __grid_constant__ CUtensorMap map_r,
                                                         float* __restrict__ pout, int kchunk, int* status) {
    using Tl = JTile<T>;
    constexpr int BX = Tl::BX, BY = Tl::BY, SLOTS = Tl::SLOTS, W = JB_W, EX = JB_EX, EY = JB_EY;
    constexpr int PP = JB_PLANE_PAD;
    extern __shared__ __align__(128) float smem[];
    float* in_p = smem;                     // [slot][PP]
    float* in_r = smem + SLOTS * PP;        // [slot][PP]
    float* lv = smem + 2 * SLOTS * PP;      // [t-1][plane % 3][PP], t = 1..T-1
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + (2 * SLOTS + 3 * (T - 1)) * PP);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * JB_TX + tx;

    const int x0 = blockIdx.x * BX + 1 - T;    // global i of extended column 0
    const int xa = x0 - (((x0 % 4) + 4) % 4);  // TMA x origin, multiple of 4
    const int off = x0 - xa;                   // 0..3
    const int y0 = blockIdx.y * BY + 1 - T;
    const int k0 = 1 + blockIdx.z * kchunk;
    const int k1 = min(g.nz, k0 + kchunk - 1);
    const int s_lo = max(0, k0 - T), s_end = k1 + T, s_ld = min(g.nz + 1, s_end);
    // No wall inside the extended tile: every column is interior and every
    // in-plane coefficient is the full one.
    const bool open = x0 >= 1 && x0 + EX - 1 <= g.nx && y0 >= 1 && y0 + EY - 1 <= g.ny;

    auto issue = [&](int plane, int sl) {
        mbar_arrive_expect_tx(&bar[sl], 2 * JB_BOX_BYTES);
        tma_load_3d(in_p + sl * PP, &map_p, xa, y0, plane, &bar[sl]);
        tma_load_3d(in_r + sl * PP, &map_r, xa, y0, plane, &bar[sl]);
    };
    if (tid == 0) {
        for (int q = 0; q < SLOTS; ++q) mbar_init(&bar[q], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int q = 0; q < SLOTS && s_lo + q <= s_ld; ++q) issue(s_lo + q, q);

    const float cx = g.dxi * g.dxi, cy = g.dyi * g.dyi, cz = g.dzi * g.dzi;
    // Diagonal of a column with no in-plane wall: interior planes, first
    // plane, last plane (reference operand order), and IEEE reciprocals.
    auto ap_open = [&](int k) {
        const float af = (k != g.nz) ? cz : 0.0f;
        const float ab = (k != 1) ? cz : 0.0f;
        return -(cx + cx + cy + cy + af + ab);
    };
    const float apm = ap_open(2), ap1 = ap_open(1), apn = ap_open(g.nz);
    const float rpm = __frcp_rn(apm), rp1 = __frcp_rn(ap1), rpn = __frcp_rn(apn);

    // slot[d] = ring slot of input plane s - d (d = 0..HOLD+1), kept
    // incrementally; the first use of every slot has parity 0.
    int slot[T + 3];
#pragma unroll
    for (int d = 0; d < T + 3; ++d) slot[d] = (((s_lo - d - s_lo) % SLOTS) + SLOTS) % SLOTS;
    uint32_t par_bits = 0;  // bit q: parity of the next wait on slot q
    int s3 = s_lo % 3;      // s mod 3 for the level rings

    bool ok = true;
    // Level t is needed at planes k0-(T-t) .. k1+(T-t) and is produced at
    // step s = plane + t; input planes exist up to the ghost plane nz+1.
    for (int s = s_lo; s <= s_end; ++s) {
        if (s <= s_ld) {
            ok &= mbar_wait(&bar[slot[0]], (par_bits >> slot[0]) & 1u);
            par_bits ^= 1u << slot[0];
        }
#pragma unroll
        for (int t = 1; t <= T; ++t) {
            const int q = s - t;  // plane of level t
            const int lo = k0 - (T - t), hi = k1 + (T - t);
            if (q >= max(0, lo) && q <= min(g.nz + 1, hi)) {
                // rings of level t-1 (t >= 2): plane x sits at x % 3
                const int rq = (s3 - t + 6) % 3, rm = (s3 - t + 5) % 3, rp = (s3 - t + 7) % 3;
                const float* Pm = (t == 1) ? in_p + slot[2] * PP : lv + ((t - 2) * 3 + rm) * PP;
                const float* Pc = (t == 1) ? in_p + slot[1] * PP : lv + ((t - 2) * 3 + rq) * PP;
                const float* Pp = (t == 1) ? in_p + slot[0] * PP : lv + ((t - 2) * 3 + rp) * PP;
                const float* Rq = in_r + slot[t] * PP;
                float* Out = lv + ((t < T ? t - 1 : 0) * 3 + rq) * PP;
                const bool zin = q >= 1 && q <= g.nz;
                const float af = (q != g.nz) ? cz : 0.0f;
                const float ab = (q != 1) ? cz : 0.0f;
                const float apo = (q == 1) ? ap1 : ((q == g.nz) ? apn : apm);
                const float rapo = (q == 1) ? rp1 : ((q == g.nz) ? rpn : rpm);
                const int ex = t + tx;
                const int gi = x0 + ex;
                if (ex < EX - t) {
#pragma unroll
                    for (int r = 0; r < JB_ROWS; ++r) {
                        const int ey = t + ty + r * JB_TY;
                        if (ey < EY - t) {
                            const int c = ey * W + ex + off;
                            const int gj = y0 + ey;
                            float val = Pc[c];  // ghosts and cells outside the box carry over
                            bool upd = false;
                            if (open) {
                                if (zin) {
                                    val = div_rn_pre(Rq[c] - cx * Pc[c + 1] - cx * Pc[c - 1] - cy * Pc[c + W] -
                                                         cy * Pc[c - W] - af * Pp[c] - ab * Pm[c],
                                                     apo, rapo);
                                    upd = true;
                                }
                            } else if (zin && gi >= 1 && gi <= g.nx && gj >= 1 && gj <= g.ny) {
                                const float ae = (gi != g.nx) ? cx : 0.0f;
                                const float aw = (gi != 1) ? cx : 0.0f;
                                const float an = (gj != g.ny) ? cy : 0.0f;
                                const float as = (gj != 1) ? cy : 0.0f;
                                const float ap = -(ae + aw + an + as + af + ab);
                                val = div_rn_pre(Rq[c] - ae * Pc[c + 1] - aw * Pc[c - 1] - an * Pc[c + W] -
                                                     as * Pc[c - W] - af * Pp[c] - ab * Pm[c],
                                                 ap, __frcp_rn(ap));
                                upd = true;
                            }
                            if (t < T) {
                                Out[c] = val;
                            } else if (upd && q >= k0 && q <= k1) {
                                pout[gidx(g, gi, gj, q)] = val;
                            }
                        }
                    }
                }
            }
            __syncthreads();
        }
        // The slot of plane s - HOLD is no longer read: refill it.
        const int freed = s - Tl::HOLD;
        if (tid == 0 && freed >= s_lo && freed + SLOTS <= s_ld) {
            fence_proxy_async_smem();
            issue(freed + SLOTS, slot[Tl::HOLD]);
        }
#pragma unroll
        for (int d = T + 2; d > 0; --d) slot[d] = slot[d - 1];
        slot[0] = (slot[0] + 1 == SLOTS) ? 0 : slot[0] + 1;
        s3 = (s3 == 2) ? 0 : s3 + 1;
    }
    if (!ok) {
        // A load that did not land in time may still be in flight: wait
        // (bounded) for the last planes issued before leaving.
        for (int pl = max(s_lo, s_ld - SLOTS + 1); pl <= s_ld; ++pl) {
            const int sl = (pl - s_lo) % SLOTS;
            mbar_wait(&bar[sl], (par_bits >> sl) & 1u);
        }
        atomicOr(status, DEV_TMA_TIMEOUT);
    }
    (void)BX;
    (void)BY;
}

// ---- one sweep streaming along z (no TMA, no temporal blocking) -------------
// A block owns 32 x 8 columns and a chunk of planes.  A thread keeps its
// column's p(k-1), p(k), p(k+1) in registers; the block shares plane k with a
// one-cell in-plane halo through shared memory, double-buffered by plane
// parity (one barrier per plane).  The loads of the next plane (its own cell
// two planes up, its halo cells and rhs one plane up) are issued a plane
// ahead.  Same per-cell expression and operand order as k_jacobi_tb.
//
// Selected with VOF_JACOBI=col.  Measured on a B200: faster than the blocked
// kernel on small grids (64^3 0.088 vs 0.103 ms per plain step), slower from
// about 128^3 up (200^3: 41 vs 34.6 us per sweep); the paired kernel below
// (no shared memory, no barrier) beats both at every size.
constexpr int JC_TX = 32, JC_TY = 8;
__global__ void __launch_bounds__(JC_TX * JC_TY) k_jacobi_col(Geom g, const float* __restrict__ pin,
                                                             const float* __restrict__ rhs,
                                                             float* __restrict__ pout, int kchunk) {
    __shared__ float sp[2][JC_TY + 2][JC_TX + 2];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = 1 + blockIdx.x * JC_TX + tx, j = 1 + blockIdx.y * JC_TY + ty;
    const int k0 = 1 + blockIdx.z * kchunk, k1 = min(g.nz, k0 + kchunk - 1);
    const bool act = i <= g.nx && j <= g.ny;
    // loads stay inside the field (the ghost layer at nx+1, ny+1 exists)
    const int il = min(i, g.nx + 1), jl = min(j, g.ny + 1);
    const int plane = g.plane;
    const int c = gidx(g, il, jl, 0);
    // this thread's halo cell of the tile, if any: x-, x+, y-, y+ edge
    int hoff = -1, hs = 0;
    if (tx == 0) { hoff = gidx(g, il - 1, jl, 0); hs = (ty + 1) * (JC_TX + 2); }
    else if (tx == JC_TX - 1) { hoff = gidx(g, min(il + 1, g.nx + 1), jl, 0); hs = (ty + 1) * (JC_TX + 2) + JC_TX + 1; }
    int voff = -1, vs = 0;  // y halo (threads of the first and last row)
    if (ty == 0) { voff = gidx(g, il, jl - 1, 0); vs = tx + 1; }
    else if (ty == JC_TY - 1) { voff = gidx(g, il, min(jl + 1, g.ny + 1), 0); vs = (JC_TY + 1) * (JC_TX + 2) + tx + 1; }
    const int own = (ty + 1) * (JC_TX + 2) + tx + 1;

    const float cx = g.dxi * g.dxi, cy = g.dyi * g.dyi, cz = g.dzi * g.dzi;
    const float ae = (i != g.nx) ? cx : 0.0f, aw = (i != 1) ? cx : 0.0f;
    const float an = (j != g.ny) ? cy : 0.0f, as = (j != 1) ? cy : 0.0f;
    // diagonal and IEEE reciprocal by plane class: interior, first, last, both
    const float ap0 = -(ae + aw + an + as + cz + cz), ap1 = -(ae + aw + an + as + cz + 0.0f);
    const float ap2 = -(ae + aw + an + as + 0.0f + cz), ap3 = -(ae + aw + an + as + 0.0f + 0.0f);
    const float rap0 = __frcp_rn(ap0), rap1 = __frcp_rn(ap1), rap2 = __frcp_rn(ap2), rap3 = __frcp_rn(ap3);
    float pm = pin[c + (k0 - 1) * plane], pc = pin[c + k0 * plane], pp = pin[c + (k0 + 1) * plane];
    float hc = hoff >= 0 ? pin[hoff + k0 * plane] : 0.0f, vc = voff >= 0 ? pin[voff + k0 * plane] : 0.0f;
    float rc = rhs[c + k0 * plane];
    for (int k = k0; k <= k1; ++k) {
        float* t = &sp[k & 1][0][0];
        t[own] = pc;
        if (hoff >= 0) t[hs] = hc;
        if (voff >= 0) t[vs] = vc;
        // next plane's operands
        const bool more = k < k1;
        const float pq = (more && k + 2 <= g.nz + 1) ? pin[c + (k + 2) * plane] : 0.0f;
        const float hn = (more && hoff >= 0) ? pin[hoff + (k + 1) * plane] : 0.0f;
        const float vn = (more && voff >= 0) ? pin[voff + (k + 1) * plane] : 0.0f;
        const float rn = more ? rhs[c + (k + 1) * plane] : 0.0f;
        __syncthreads();
        if (act) {
            const bool kb = k == 1, kt = k == g.nz;
            const float ap = kb ? (kt ? ap3 : ap1) : (kt ? ap2 : ap0);
            const float rap = kb ? (kt ? rap3 : rap1) : (kt ? rap2 : rap0);
            const float af = (k != g.nz) ? cz : 0.0f, ab = (k != 1) ? cz : 0.0f;
            const float pE = t[own + 1], pW = t[own - 1], pN = t[own + JC_TX + 2], pS = t[own - (JC_TX + 2)];
            pout[c + k * plane] =
                div_rn_pre(rc - ae * pE - aw * pW - an * pN - as * pS - af * pp - ab * pm, ap, rap);
        }
        pm = pc;
        pc = pp;
        pp = pq;
        hc = hn;
        vc = vn;
        rc = rn;
    }
}

cudaError_t jacobi_col_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s) {
    const int bx = (g.nx + JC_TX - 1) / JC_TX, by = (g.ny + JC_TY - 1) / JC_TY;
    const int target = (int)((long long)g.nz * bx * by / 600);
    const int len = target < 1 ? 1 : (target > 16 ? 16 : target);
    const int nch = (g.nz + len - 1) / len, kchunk = (g.nz + nch - 1) / nch;
    k_jacobi_col<<<dim3(bx, by, (g.nz + kchunk - 1) / kchunk), dim3(JC_TX, JC_TY), 0, s>>>(g, pin, rhs, pout,
                                                                                         kchunk);
    return cudaGetLastError();
}

// ---- one sweep, two cells per thread, streaming along z ---------------------
// Cells are paired by padded column (2m, 2m + 1): pair m of a row is one
// aligned 8-byte word (px is a multiple of 32).  The pairs of rows 1..ny are
// numbered flat, q = (j - 1) npair + m, and 32 consecutive pairs make a warp
// across row ends, so every lane has work at every width.  A thread marches
// kchunk planes with its pair's p(k - 1), p(k), p(k + 1) in registers; the y
// neighbours are loads (served by L1), the x neighbours come from the
// neighbouring lanes, or from memory at the ends of a warp and of a row; the
// next plane's operands are loaded a plane ahead; no shared memory, no
// barrier.  Each cell's update is the scalar expression of k_jacobi_tb, in the
// same operand order.  (The packed f32x2 instructions are not used here: in a
// chain of them the code generator fuses a product into the following
// subtraction, which changes the rounding; a probe on a B200 found a quarter
// of such two-term chains off by an ulp even with .rn on every instruction.)
// The ghost cell of a pair (column 0 or nx + 1) is never stored.
constexpr int JP_THREADS = 256;

__global__ void __launch_bounds__(JP_THREADS) k_jacobi_pairs(Geom g, const float* __restrict__ pin,
                                                             const float* __restrict__ rhs,
                                                             float* __restrict__ pout, int kchunk) {
    const int npair = g.nx / 2 + 1;  // pairs covering columns 0 .. nx
    const int nq = npair * g.ny;
    const int qt = blockIdx.x * JP_THREADS + threadIdx.x;
    const bool qa = qt < nq;
    const int q = qa ? qt : nq - 1;  // lanes past the end shadow the last pair
    const int jr = q / npair, m = q - jr * npair;
    const int j = jr + 1, i0 = 2 * m, i1 = i0 + 1;
    const bool a0 = qa && i0 >= 1, a1 = qa && i1 <= g.nx;
    const int lane = threadIdx.x & 31;
    const bool ldw = lane == 0 && m > 0;             // x- neighbour of cell i0 from memory
    const bool lde = lane == 31 || m == npair - 1;   // x+ neighbour of cell i1 from memory
    const int k0 = 1 + blockIdx.y * kchunk, k1 = min(g.nz, k0 + kchunk - 1);
    const int plane = g.plane;
    const int c = gidx(g, i0, j, 0);  // even
    const int cw = c - 1, ce = c + min(2, g.px - 1 - i0);
    const float cx = g.dxi * g.dxi, cy = g.dyi * g.dyi, cz = g.dzi * g.dzi;
    const float ae0 = (i0 != g.nx) ? cx : 0.0f, aw0 = (i0 != 1) ? cx : 0.0f;
    const float ae1 = (i1 != g.nx) ? cx : 0.0f, aw1 = (i1 != 1) ? cx : 0.0f;
    const float an = (j != g.ny) ? cy : 0.0f, as = (j != 1) ? cy : 0.0f;
    // diagonal of an inner plane in the reference's operand order and its IEEE
    // reciprocal (the first and last planes compute theirs when they come)
    const float2 dm = make_float2(-(ae0 + aw0 + an + as + cz + cz), -(ae1 + aw1 + an + as + cz + cz));
    const float2 rm = make_float2(__frcp_rn(dm.x), __frcp_rn(dm.y));
    const float2* P = reinterpret_cast<const float2*>(pin);
    const float2* R = reinterpret_cast<const float2*>(rhs);
    float2* O = reinterpret_cast<float2*>(pout);
    const int w = c >> 1, wp = plane >> 1, wr = g.px >> 1;
    const float2 zero = make_float2(0.0f, 0.0f);
    float2 pm = P[w + (k0 - 1) * wp], pc = P[w + k0 * wp], pp = P[w + (k0 + 1) * wp];
    float2 pS = P[w + k0 * wp - wr], pN = P[w + k0 * wp + wr], rc = R[w + k0 * wp];
    float xw = ldw ? pin[cw + k0 * plane] : 0.0f, xe = lde ? pin[ce + k0 * plane] : 0.0f;
    for (int k = k0; k <= k1; ++k) {
        // operands of the next plane
        const bool more = k < k1;
        const float2 pq = (more && k + 2 <= g.nz + 1) ? P[w + (k + 2) * wp] : zero;
        const float2 sn = more ? P[w + (k + 1) * wp - wr] : zero;
        const float2 nn = more ? P[w + (k + 1) * wp + wr] : zero;
        const float2 rn = more ? R[w + (k + 1) * wp] : zero;
        const float xwn = (more && ldw) ? pin[cw + (k + 1) * plane] : 0.0f;
        const float xen = (more && lde) ? pin[ce + (k + 1) * plane] : 0.0f;
        float pw = __shfl_up_sync(0xffffffffu, pc.y, 1), pe = __shfl_down_sync(0xffffffffu, pc.x, 1);
        if (ldw) pw = xw;
        if (lde) pe = xe;
        const bool kb = k == 1, kt = k == g.nz;
        const float af = kt ? 0.0f : cz, ab = kb ? 0.0f : cz;
        float2 d = dm, rd = rm;
        if (kb || kt) {
            d = make_float2(-(ae0 + aw0 + an + as + af + ab), -(ae1 + aw1 + an + as + af + ab));
            rd = make_float2(__frcp_rn(d.x), __frcp_rn(d.y));
        }
        const float v0 =
            div_rn_pre(rc.x - ae0 * pc.y - aw0 * pw - an * pN.x - as * pS.x - af * pp.x - ab * pm.x, d.x, rd.x);
        const float v1 =
            div_rn_pre(rc.y - ae1 * pe - aw1 * pc.x - an * pN.y - as * pS.y - af * pp.y - ab * pm.y, d.y, rd.y);
        const int o = w + k * wp;
        if (a0 && a1)
            O[o] = make_float2(v0, v1);
        else if (a0)
            pout[2 * o] = v0;
        else if (a1)
            pout[2 * o + 1] = v1;
        pm = pc;
        pc = pp;
        pp = pq;
        pS = sn;
        pN = nn;
        rc = rn;
        xw = xwn;
        xe = xen;
    }
}

// ---- the paired sweep with the plane cases peeled out of the march -----------
// k_jacobi_pairs evaluates, on every plane, whether there is a next plane to
// load (zeros otherwise) and whether the plane is a wall plane (its own
// diagonal), and copies its plane registers one place down.  Here the march
// is split: the first plane of the box (k = 1) and the last plane of the
// chunk run through the general plane step; the planes between load their
// successors unconditionally and take the inner diagonal, in a loop unrolled
// U times so that the plane registers are renamed instead of copied.  The
// per-cell expression and operand order are k_jacobi_pairs', so are the bits.
struct JPLine {
    const float2* P;
    const float2* R;
    float2* O;
    const float* pin;
    float* pout;
    int w, wp, wr, cw, ce, plane;
    float ae0, aw0, ae1, aw1, an, as, cz;
    float2 dm, rm;
    bool a0, a1, ldw, lde;
};

struct JPRegs {
    float2 pm, pc, pp, pS, pN, rc;
    float xw, xe;
};

// One plane k of the paired sweep.  MORE: load the next plane's operands (the
// caller guarantees k < k1 <= nz, so plane k + 2 <= nz + 1 exists; marching
// DOWN, k > k0 >= 1, so plane k - 2 >= 0 exists).  EDGE: the plane may be the
// first or the last of the box.  DOWN marches k downwards: the next plane is
// k - 1, and the window pm, pc, pp turns the other way; each cell's
// expression is the same.
template <bool MORE, bool EDGE, bool DOWN = false>
__device__ __forceinline__ void jp_plane(const JPLine& L, const Geom& g, int k, JPRegs& s) {
    float2 pq, sn, nn, rn;
    float xwn = 0.0f, xen = 0.0f;
    if constexpr (MORE) {
        const int kn = DOWN ? k - 1 : k + 1;
        const int o1 = L.w + kn * L.wp;
        pq = L.P[DOWN ? o1 - L.wp : o1 + L.wp];
        sn = L.P[o1 - L.wr];
        nn = L.P[o1 + L.wr];
        rn = L.R[o1];
        if (L.ldw) xwn = L.pin[L.cw + kn * L.plane];
        if (L.lde) xen = L.pin[L.ce + kn * L.plane];
    }
    float pw = __shfl_up_sync(0xffffffffu, s.pc.y, 1), pe = __shfl_down_sync(0xffffffffu, s.pc.x, 1);
    if (L.ldw) pw = s.xw;
    if (L.lde) pe = s.xe;
    float af = L.cz, ab = L.cz;
    float2 d = L.dm, rd = L.rm;
    if constexpr (EDGE) {
        const bool kb = k == 1, kt = k == g.nz;
        af = kt ? 0.0f : L.cz;
        ab = kb ? 0.0f : L.cz;
        if (kb || kt) {
            d = make_float2(-(L.ae0 + L.aw0 + L.an + L.as + af + ab), -(L.ae1 + L.aw1 + L.an + L.as + af + ab));
            rd = make_float2(__frcp_rn(d.x), __frcp_rn(d.y));
        }
    }
    const float v0 = div_rn_pre(s.rc.x - L.ae0 * s.pc.y - L.aw0 * pw - L.an * s.pN.x - L.as * s.pS.x -
                                    af * s.pp.x - ab * s.pm.x,
                                d.x, rd.x);
    const float v1 = div_rn_pre(s.rc.y - L.ae1 * pe - L.aw1 * s.pc.x - L.an * s.pN.y - L.as * s.pS.y -
                                    af * s.pp.y - ab * s.pm.y,
                                d.y, rd.y);
    const int o = L.w + k * L.wp;
    if (L.a0 && L.a1)
        L.O[o] = make_float2(v0, v1);
    else if (L.a0)
        L.pout[2 * o] = v0;
    else if (L.a1)
        L.pout[2 * o + 1] = v1;
    if constexpr (MORE) {
        if constexpr (DOWN) {
            s.pp = s.pc;
            s.pc = s.pm;
            s.pm = pq;
        } else {
            s.pm = s.pc;
            s.pc = s.pp;
            s.pp = pq;
        }
        s.pS = sn;
        s.pN = nn;
        s.rc = rn;
        s.xw = xwn;
        s.xe = xen;
    }
}

template <int U, int MINB, bool DOWN = false>
__global__ void __launch_bounds__(JP_THREADS, MINB) k_jacobi_peel(Geom g, const float* __restrict__ pin,
                                                            const float* __restrict__ rhs,
                                                            float* __restrict__ pout, int kchunk) {
    const int npair = g.nx / 2 + 1;  // pairs covering columns 0 .. nx
    const int nq = npair * g.ny;
    const int qt = blockIdx.x * JP_THREADS + threadIdx.x;
    const bool qa = qt < nq;
    const int q = qa ? qt : nq - 1;  // lanes past the end shadow the last pair
    const int jr = q / npair, m = q - jr * npair;
    const int j = jr + 1, i0 = 2 * m, i1 = i0 + 1;
    const int lane = threadIdx.x & 31;
    const int k0 = 1 + blockIdx.y * kchunk, k1 = min(g.nz, k0 + kchunk - 1);
    JPLine L;
    L.P = reinterpret_cast<const float2*>(pin);
    L.R = reinterpret_cast<const float2*>(rhs);
    L.O = reinterpret_cast<float2*>(pout);
    L.pin = pin;
    L.pout = pout;
    L.a0 = qa && i0 >= 1;
    L.a1 = qa && i1 <= g.nx;
    L.ldw = lane == 0 && m > 0;            // x- neighbour of cell i0 from memory
    L.lde = lane == 31 || m == npair - 1;  // x+ neighbour of cell i1 from memory
    L.plane = g.plane;
    const int c = gidx(g, i0, j, 0);  // even
    L.cw = c - 1;
    L.ce = c + min(2, g.px - 1 - i0);
    const float cx = g.dxi * g.dxi, cy = g.dyi * g.dyi;
    L.cz = g.dzi * g.dzi;
    L.ae0 = (i0 != g.nx) ? cx : 0.0f;
    L.aw0 = (i0 != 1) ? cx : 0.0f;
    L.ae1 = (i1 != g.nx) ? cx : 0.0f;
    L.aw1 = (i1 != 1) ? cx : 0.0f;
    L.an = (j != g.ny) ? cy : 0.0f;
    L.as = (j != 1) ? cy : 0.0f;
    L.dm = make_float2(-(L.ae0 + L.aw0 + L.an + L.as + L.cz + L.cz), -(L.ae1 + L.aw1 + L.an + L.as + L.cz + L.cz));
    L.rm = make_float2(__frcp_rn(L.dm.x), __frcp_rn(L.dm.y));
    L.w = c >> 1;
    L.wp = g.plane >> 1;
    L.wr = g.px >> 1;
    JPRegs s;
    const int ks = DOWN ? k1 : k0;  // the march's first plane
    s.pm = L.P[L.w + (ks - 1) * L.wp];
    s.pc = L.P[L.w + ks * L.wp];
    s.pp = L.P[L.w + (ks + 1) * L.wp];
    s.pS = L.P[L.w + ks * L.wp - L.wr];
    s.pN = L.P[L.w + ks * L.wp + L.wr];
    s.rc = L.R[L.w + ks * L.wp];
    s.xw = L.ldw ? pin[L.cw + ks * L.plane] : 0.0f;
    s.xe = L.lde ? pin[L.ce + ks * L.plane] : 0.0f;
    int k = ks;
    if constexpr (DOWN) {
        if (k == g.nz && k > k0) {
            jp_plane<true, true, true>(L, g, k, s);
            --k;
        }
        VOF_UNROLL(U)
        for (; k > k0; --k) jp_plane<true, false, true>(L, g, k, s);
        jp_plane<false, true, true>(L, g, k0, s);
    } else {
        if (k == 1 && k < k1) {
            jp_plane<true, true>(L, g, k, s);
            ++k;
        }
        VOF_UNROLL(U)
        for (; k < k1; ++k) jp_plane<true, false>(L, g, k, s);
        jp_plane<false, true>(L, g, k1, s);
    }
}

// VOF_JP_UNROLL (1, 2 or 4) picks the unroll of the peeled march and
// VOF_JP_MINB (1 or 4) the blocks per SM its registers are sized for.
// The downward march (the sweeps' alternating direction) is built for the
// default shape only.
using JPKernel = void (*)(Geom, const float*, const float*, float*, int);
static JPKernel jp_peel_kernel() {
    static JPKernel k = nullptr;
    if (!k) {
        const char* v = getenv("VOF_JP_UNROLL");
        const char* b = getenv("VOF_JP_MINB");
        const int u = v ? atoi(v) : 2;
        const int mb = b ? atoi(b) : 4;
        k = u == 1 ? (mb == 4 ? k_jacobi_peel<1, 4> : k_jacobi_peel<1, 1>)
            : u == 4 ? (mb == 4 ? k_jacobi_peel<4, 4> : k_jacobi_peel<4, 1>)
                     : (mb == 4 ? k_jacobi_peel<2, 4> : k_jacobi_peel<2, 1>);
    }
    return k;
}

// ---- one sweep, four cells per thread, streaming along z ---------------------
// The peeled march of k_jacobi_peel with a quad of cells per thread (i = 4m ..
// 4m + 3: one aligned 16-byte word of the padded layout; the quads of all rows
// numbered flat, so 32 consecutive quads make a warp across row ends), so that
// every load in flight carries 16 bytes instead of 8: the sweep is bound by
// memory latency at the occupancy its registers allow.  A cell's x neighbours
// are the quad's own cells, the left lane's last cell and the right lane's
// first (or memory at the ends of a warp and of a row).  The per-cell
// coefficients and inner-plane diagonals are the thread's constants; each
// cell's update is k_jacobi_pairs' expression in its operand order.
struct JQLine {
    const float4* P;
    const float4* R;
    float4* O;
    const float* pin;
    float* pout;
    int w, wp, wr, cw, ce, plane;
    int es;          // the quad's cell on an x wall (i == 1 or nx), or -1 (nx >= 4: at most one)
    bool es_e, es_w;  // ... its east (i == nx) and west (i == 1) coefficients are 0
    float cx, an, as, cz;
    float dmi, rmi;  // inner-plane diagonal and reciprocal of a cell away from the x walls
    float dms, rms;  // ... of the wall cell
    int nact0, nact1;  // the active cells are nact0 .. nact1 - 1
    bool ldw, lde;
    __device__ float ae(int e) const { return (e == es && es_e) ? 0.0f : cx; }
    __device__ float aw(int e) const { return (e == es && es_w) ? 0.0f : cx; }
    __device__ bool act(int e) const { return e >= nact0 && e < nact1; }
};

struct JQRegs {
    float4 pm, pc, pp, rc;
    float xw, xe;
};

__device__ __forceinline__ float q4(const float4& v, int e) {
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

template <bool MORE, bool EDGE>
__device__ __forceinline__ void jq_plane(const JQLine& L, const Geom& g, int k, JQRegs& s) {
    float4 pq, rn;
    float xwn = 0.0f, xen = 0.0f;
    // the y neighbours of this plane (L1 / L2: the rows of other warps)
    const float4 pS = L.P[L.w + k * L.wp - L.wr], pN = L.P[L.w + k * L.wp + L.wr];
    if constexpr (MORE) {
        const int o1 = L.w + (k + 1) * L.wp;
        pq = L.P[o1 + L.wp];
        rn = L.R[o1];
        if (L.ldw) xwn = L.pin[L.cw + (k + 1) * L.plane];
        if (L.lde) xen = L.pin[L.ce + (k + 1) * L.plane];
    }
    float pw = __shfl_up_sync(0xffffffffu, s.pc.w, 1), pe = __shfl_down_sync(0xffffffffu, s.pc.x, 1);
    if (L.ldw) pw = s.xw;
    if (L.lde) pe = s.xe;
    float af = L.cz, ab = L.cz;
    bool wall = false;
    if constexpr (EDGE) {
        const bool kb = k == 1, kt = k == g.nz;
        af = kt ? 0.0f : L.cz;
        ab = kb ? 0.0f : L.cz;
        wall = kb || kt;
    }
    float v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float ae = L.ae(e), aw = L.aw(e);
        float d = (e == L.es) ? L.dms : L.dmi, rd = (e == L.es) ? L.rms : L.rmi;
        if (EDGE && wall) {
            d = -(ae + aw + L.an + L.as + af + ab);
            rd = __frcp_rn(d);
        }
        const float pE = e == 3 ? pe : q4(s.pc, e + 1), pW = e == 0 ? pw : q4(s.pc, e - 1);
        v[e] = div_rn_pre(q4(s.rc, e) - ae * pE - aw * pW - L.an * q4(pN, e) - L.as * q4(pS, e) -
                              af * q4(s.pp, e) - ab * q4(s.pm, e),
                          d, rd);
    }
    const int o = L.w + k * L.wp;
    if (L.nact0 == 0 && L.nact1 == 4) {
        L.O[o] = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (L.act(e)) L.pout[4 * o + e] = v[e];
    }
    if constexpr (MORE) {
        s.pm = s.pc;
        s.pc = s.pp;
        s.pp = pq;
        s.rc = rn;
        s.xw = xwn;
        s.xe = xen;
    }
}

__global__ void __launch_bounds__(256, 3) k_jacobi_quad(Geom g, const float* __restrict__ pin,
                                                        const float* __restrict__ rhs, float* __restrict__ pout,
                                                        int kchunk) {
    const int nquad = g.nx / 4 + 1;  // quads covering columns 0 .. nx
    const int nq = nquad * g.ny;
    const int qt = blockIdx.x * blockDim.x + threadIdx.x;
    const bool qa = qt < nq;
    const int q = qa ? qt : nq - 1;  // lanes past the end shadow the last quad
    const int jr = q / nquad, m = q - jr * nquad;
    const int j = jr + 1, i0 = 4 * m;
    const int lane = threadIdx.x & 31;
    const int k0 = 1 + blockIdx.y * kchunk, k1 = min(g.nz, k0 + kchunk - 1);
    JQLine L;
    L.P = reinterpret_cast<const float4*>(pin);
    L.R = reinterpret_cast<const float4*>(rhs);
    L.O = reinterpret_cast<float4*>(pout);
    L.pin = pin;
    L.pout = pout;
    L.ldw = lane == 0 && m > 0;            // x- neighbour of the first cell from memory
    L.lde = lane == 31 || m == nquad - 1;  // x+ neighbour of the last cell from memory
    L.plane = g.plane;
    const int c = gidx(g, i0, j, 0);  // a multiple of 4
    L.cw = c - 1;
    L.ce = c + 4;  // i0 + 4 <= nx + 3 < px: within the row
    const float cy = g.dyi * g.dyi;
    L.cx = g.dxi * g.dxi;
    L.cz = g.dzi * g.dzi;
    L.an = (j != g.ny) ? cy : 0.0f;
    L.as = (j != 1) ? cy : 0.0f;
    L.es = (i0 <= 1 && 1 <= i0 + 3) ? 1 - i0 : ((i0 <= g.nx && g.nx <= i0 + 3) ? g.nx - i0 : -1);
    L.es_w = L.es >= 0 && i0 + L.es == 1;
    L.es_e = L.es >= 0 && i0 + L.es == g.nx;
    L.dmi = -(L.cx + L.cx + L.an + L.as + L.cz + L.cz);
    L.rmi = __frcp_rn(L.dmi);
    {
        const float ae = L.es_e ? 0.0f : L.cx, aw = L.es_w ? 0.0f : L.cx;
        L.dms = -(ae + aw + L.an + L.as + L.cz + L.cz);
        L.rms = __frcp_rn(L.dms);
    }
    L.nact0 = qa ? max(0, 1 - i0) : 4;
    L.nact1 = qa ? min(4, g.nx + 1 - i0) : 4;
    L.w = c >> 2;
    L.wp = g.plane >> 2;
    L.wr = g.px >> 2;
    JQRegs s;
    s.pm = L.P[L.w + (k0 - 1) * L.wp];
    s.pc = L.P[L.w + k0 * L.wp];
    s.pp = L.P[L.w + (k0 + 1) * L.wp];
    s.rc = L.R[L.w + k0 * L.wp];
    s.xw = L.ldw ? pin[L.cw + k0 * L.plane] : 0.0f;
    s.xe = L.lde ? pin[L.ce + k0 * L.plane] : 0.0f;
    int k = k0;
    if (k == 1 && k < k1) {
        jq_plane<true, true>(L, g, k, s);
        ++k;
    }
    for (; k < k1; ++k) jq_plane<true, false>(L, g, k, s);
    jq_plane<false, true>(L, g, k1, s);
}

// ---- the paired sweep fed by bulk copies of whole rows ------------------------
// A block owns BY rows of the grid (whole padded rows, x complete) and a
// chunk of planes.  One producer thread (the last warp's lane 0) streams, for
// every plane k0-1 .. k1+1, the BY + 2 pressure rows j0-1 .. j0+BY and, for
// the block's own planes, the BY rhs rows into a ring of JS_SLOTS
// shared-memory slots with untiled bulk copies (cp.async.bulk; the rows of a
// plane are contiguous, so one copy per field and plane, completing on the
// slot's "full" mbarrier), up to JS_SLOTS planes ahead.  The consumer threads
// own one pair of cells (i0 = 2m, i1 = i0 + 1) of one row each; at plane k
// they read the pair and its x and y neighbours from plane k's slot, the
// planes above and below from the slots beside it (the pair's own column of
// plane k - 1 and k from registers), evaluate k_jacobi_pairs' per-cell
// expression in its operand order (same bits), store the pair, and each warp
// marks plane k's slot "empty" for the producer.  No register holds a
// load in flight, so the bytes in flight are the ring's, not the occupancy's.
// Every wait is bounded: a wait that runs out sets DEV_TMA_TIMEOUT in the
// status word and ends the loop; the producer then waits (bounded) for the
// copies it issued before the block exits.
constexpr int JS_SLOTS = 8;

template <int BY>
__global__ void __launch_bounds__(512, 3) k_jacobi_bulk(Geom g, const float* __restrict__ pin,
                                                      const float* __restrict__ rhs, float* __restrict__ pout,
                                                      int kchunk, int* status) {
    constexpr int slots = JS_SLOTS;
    extern __shared__ __align__(128) unsigned char js_smem[];
    const int px = g.px;
    const int slot_floats = (2 * BY + 2) * px;  // BY + 2 pressure rows, BY rhs rows
    float* ring = reinterpret_cast<float*>(js_smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(js_smem + (size_t)slots * slot_floats * sizeof(float));
    uint64_t* empty = full + JS_SLOTS;
    const int ncw = ((int)blockDim.x >> 5) - 1;  // consumer warps
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j0 = 1 + blockIdx.x * BY;
    const int nrow = min(BY, g.ny - j0 + 1);
    const int k0 = 1 + blockIdx.y * kchunk, k1 = min(g.nz, k0 + kchunk - 1);
    const int nplanes = k1 - k0 + 3;  // planes k0 - 1 .. k1 + 1
    if (threadIdx.x == 0) {
        for (int s = 0; s < slots; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], ncw);
        }
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == ncw) {  // producer
        if (lane != 0) return;
        const uint32_t rowb = (uint32_t)px * sizeof(float);
        bool ok = true;
        int issued = 0;
        for (int n = 0; n < nplanes; ++n) {
            const int s = n % slots;
            if (n >= slots && !(ok = mbar_wait(&empty[s], (uint32_t)((n / slots - 1) & 1)))) break;
            const int kk = k0 - 1 + n;
            const bool own = kk >= k0 && kk <= k1;
            float* dst = ring + (size_t)s * slot_floats;
            mbar_arrive_expect_tx(&full[s], rowb * (uint32_t)(nrow + 2 + (own ? nrow : 0)));
            bulk_load(dst, pin + gidx(g, 0, j0 - 1, kk), rowb * (uint32_t)(nrow + 2), &full[s]);
            if (own) bulk_load(dst + (BY + 2) * px, rhs + gidx(g, 0, j0, kk), rowb * (uint32_t)nrow, &full[s]);
            issued = n + 1;
        }
        if (!ok) {
            atomicOr(status, DEV_TMA_TIMEOUT);
            // no copy may outlive the block: wait for the last fill of every slot
            for (int n = issued - 1; n >= 0 && n >= issued - slots; --n)
                mbar_wait(&full[n % slots], (uint32_t)((n / slots) & 1));
        }
        return;
    }

    // consumers: one pair per thread
    const int npair = g.nx / 2 + 1;
    const int t = threadIdx.x;
    const bool act = t < nrow * npair;
    const int r = act ? t / npair : 0, m = act ? t - r * npair : 0;
    const int j = j0 + r, i0 = 2 * m, i1 = i0 + 1;
    const bool a0 = act && i0 >= 1, a1 = act && i1 <= g.nx;
    const float cx = g.dxi * g.dxi, cy = g.dyi * g.dyi, cz = g.dzi * g.dzi;
    const float ae0 = (i0 != g.nx) ? cx : 0.0f, aw0 = (i0 != 1) ? cx : 0.0f;
    const float ae1 = (i1 != g.nx) ? cx : 0.0f, aw1 = (i1 != 1) ? cx : 0.0f;
    const float an = (j != g.ny) ? cy : 0.0f, as = (j != 1) ? cy : 0.0f;
    const float2 dm = make_float2(-(ae0 + aw0 + an + as + cz + cz), -(ae1 + aw1 + an + as + cz + cz));
    const float2 rm = make_float2(__frcp_rn(dm.x), __frcp_rn(dm.y));
    const int off = (r + 1) * px + i0;     // the pair in a slot's pressure rows (even: float2-aligned)
    const int roff = (BY + 2 + r) * px + i0;  // ... and in its rhs rows
    float2* O = reinterpret_cast<float2*>(pout);
    const int o0 = gidx(g, i0, j, 0) >> 1;
    const int wp = g.plane >> 1;
    bool ok = mbar_wait(&full[0], 0) && mbar_wait(&full[1], 0);
    float2 pm = make_float2(0.0f, 0.0f), pc = pm;
    if (ok) {
        pm = *reinterpret_cast<const float2*>(ring + off);
        pc = *reinterpret_cast<const float2*>(ring + (size_t)slot_floats + off);
        // plane k0 - 1 is read by nobody any more (the pair's own column is in pm)
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[0]);
    }
    for (int k = k0; k <= k1 && ok; ++k) {
        const int n = k - k0 + 2;  // plane k + 1
        if (!(ok = mbar_wait(&full[n % slots], (uint32_t)((n / slots) & 1)))) break;
        const float* Pc = ring + (size_t)((n - 1) % slots) * slot_floats;
        const float* Pp = ring + (size_t)(n % slots) * slot_floats;
        const float2 pp = *reinterpret_cast<const float2*>(Pp + off);
        const float2 pN = *reinterpret_cast<const float2*>(Pc + off + px);
        const float2 pS = *reinterpret_cast<const float2*>(Pc + off - px);
        const float2 rc = *reinterpret_cast<const float2*>(Pc + roff);
        const float pw = Pc[off - 1], pe = Pc[off + 2];
        const bool kb = k == 1, kt = k == g.nz;
        const float af = kt ? 0.0f : cz, ab = kb ? 0.0f : cz;
        float2 d = dm, rd = rm;
        if (kb || kt) {
            d = make_float2(-(ae0 + aw0 + an + as + af + ab), -(ae1 + aw1 + an + as + af + ab));
            rd = make_float2(__frcp_rn(d.x), __frcp_rn(d.y));
        }
        const float v0 =
            div_rn_pre(rc.x - ae0 * pc.y - aw0 * pw - an * pN.x - as * pS.x - af * pp.x - ab * pm.x, d.x, rd.x);
        const float v1 =
            div_rn_pre(rc.y - ae1 * pe - aw1 * pc.x - an * pN.y - as * pS.y - af * pp.y - ab * pm.y, d.y, rd.y);
        const int o = o0 + k * wp;
        if (a0 && a1)
            O[o] = make_float2(v0, v1);
        else if (a0)
            pout[2 * o] = v0;
        else if (a1)
            pout[2 * o + 1] = v1;
        pm = pc;
        pc = pp;
        // plane k is read by nobody any more (its column goes on in pm)
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[(n - 1) % slots]);
    }
    if (!ok && lane == 0) atomicOr(status, DEV_TMA_TIMEOUT);
}

// ---- the paired sweep with a deeper prefetch of its own column ---------------
// k_jacobi_pairs keeps one plane of loads in flight per thread, which at
// 200^3 leaves the sweep waiting on memory (about a third of the bytes in
// flight that hide HBM latency at its occupancy).  Here each thread copies
// its own column's pressure (JR_AHEAD + 1 planes ahead) and right-hand side
// (JR_AHEAD planes ahead) into a ring of shared-memory slots of its own with
// asynchronous copies (cp.async, cached in L1 on the way, where the other
// rows' threads find them as their y neighbours), so JR_AHEAD planes of those
// loads are in flight without holding registers; a thread reads only slots it
// filled, so no barrier is needed.  Everything else -- the x neighbours by
// shuffle, the y neighbours as loads one plane ahead, the per-cell expression
// -- is k_jacobi_pairs', so the bits are the same.
constexpr int JR_AHEAD = 4, JR_SLOTS = JR_AHEAD + 1;

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem_dst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(JP_THREADS) k_jacobi_ring(Geom g, const float* __restrict__ pin,
                                                            const float* __restrict__ rhs,
                                                            float* __restrict__ pout, int kchunk) {
    __shared__ float2 ringP[JR_SLOTS][JP_THREADS];
    __shared__ float2 ringR[JR_SLOTS][JP_THREADS];
    const int npair = g.nx / 2 + 1;  // pairs covering columns 0 .. nx
    const int nq = npair * g.ny;
    const int t = threadIdx.x;
    const int qt = blockIdx.x * JP_THREADS + t;
    const bool qa = qt < nq;
    const int q = qa ? qt : nq - 1;  // lanes past the end shadow the last pair
    const int jr = q / npair, m = q - jr * npair;
    const int j = jr + 1, i0 = 2 * m, i1 = i0 + 1;
    const bool a0 = qa && i0 >= 1, a1 = qa && i1 <= g.nx;
    const int lane = t & 31;
    const bool ldw = lane == 0 && m > 0;             // x- neighbour of cell i0 from memory
    const bool lde = lane == 31 || m == npair - 1;   // x+ neighbour of cell i1 from memory
    const int k0 = 1 + blockIdx.y * kchunk, k1 = min(g.nz, k0 + kchunk - 1);
    const int plane = g.plane;
    const int c = gidx(g, i0, j, 0);  // even
    const int cw = c - 1, ce = c + min(2, g.px - 1 - i0);
    const float cx = g.dxi * g.dxi, cy = g.dyi * g.dyi, cz = g.dzi * g.dzi;
    const float ae0 = (i0 != g.nx) ? cx : 0.0f, aw0 = (i0 != 1) ? cx : 0.0f;
    const float ae1 = (i1 != g.nx) ? cx : 0.0f, aw1 = (i1 != 1) ? cx : 0.0f;
    const float an = (j != g.ny) ? cy : 0.0f, as = (j != 1) ? cy : 0.0f;
    const float2 dm = make_float2(-(ae0 + aw0 + an + as + cz + cz), -(ae1 + aw1 + an + as + cz + cz));
    const float2 rm = make_float2(__frcp_rn(dm.x), __frcp_rn(dm.y));
    const float2* P = reinterpret_cast<const float2*>(pin);
    const float2* R = reinterpret_cast<const float2*>(rhs);
    float2* O = reinterpret_cast<float2*>(pout);
    const int w = c >> 1, wp = plane >> 1, wr = g.px >> 1;
    const float2 zero = make_float2(0.0f, 0.0f);
    // group gi (issued at iteration gi, or before the loop for gi < k0)
    // copies the pressure of plane gi + JR_AHEAD + 1 and the rhs of plane
    // gi + JR_AHEAD, which iteration gi + JR_AHEAD - 1 takes as the next
    // plane's operands; planes nobody needs are not copied (empty group)
    int slot_issue = 0, slot_use = 0;
    auto issue = [&](int gi) {
        const int kp = gi + JR_AHEAD + 1, kr = gi + JR_AHEAD;
        if (kr - 1 < k1) {
            if (kp <= g.nz + 1) cp_async8(&ringP[slot_issue][t], P + w + kp * wp);
            cp_async8(&ringR[slot_issue][t], R + w + kr * wp);
        }
        cp_async_commit();
        slot_issue = slot_issue + 1 == JR_SLOTS ? 0 : slot_issue + 1;
    };
    for (int gi = k0 + 1 - JR_AHEAD; gi < k0; ++gi) issue(gi);
    float2 pm = P[w + (k0 - 1) * wp], pc = P[w + k0 * wp], pp = P[w + (k0 + 1) * wp];
    float2 pS = P[w + k0 * wp - wr], pN = P[w + k0 * wp + wr], rc = R[w + k0 * wp];
    float xw = ldw ? pin[cw + k0 * plane] : 0.0f, xe = lde ? pin[ce + k0 * plane] : 0.0f;
    for (int k = k0; k <= k1; ++k) {
        issue(k);
        // operands of the next plane
        const bool more = k < k1;
        cp_async_wait<JR_AHEAD - 1>();  // the group of iteration k + 1 - JR_AHEAD has landed
        const float2 pq = (more && k + 2 <= g.nz + 1) ? ringP[slot_use][t] : zero;
        const float2 rn = more ? ringR[slot_use][t] : zero;
        slot_use = slot_use + 1 == JR_SLOTS ? 0 : slot_use + 1;
        const float2 sn = more ? P[w + (k + 1) * wp - wr] : zero;
        const float2 nn = more ? P[w + (k + 1) * wp + wr] : zero;
        const float xwn = (more && ldw) ? pin[cw + (k + 1) * plane] : 0.0f;
        const float xen = (more && lde) ? pin[ce + (k + 1) * plane] : 0.0f;
        float pw = __shfl_up_sync(0xffffffffu, pc.y, 1), pe = __shfl_down_sync(0xffffffffu, pc.x, 1);
        if (ldw) pw = xw;
        if (lde) pe = xe;
        const bool kb = k == 1, kt = k == g.nz;
        const float af = kt ? 0.0f : cz, ab = kb ? 0.0f : cz;
        float2 d = dm, rd = rm;
        if (kb || kt) {
            d = make_float2(-(ae0 + aw0 + an + as + af + ab), -(ae1 + aw1 + an + as + af + ab));
            rd = make_float2(__frcp_rn(d.x), __frcp_rn(d.y));
        }
        const float v0 =
            div_rn_pre(rc.x - ae0 * pc.y - aw0 * pw - an * pN.x - as * pS.x - af * pp.x - ab * pm.x, d.x, rd.x);
        const float v1 =
            div_rn_pre(rc.y - ae1 * pe - aw1 * pc.x - an * pN.y - as * pS.y - af * pp.y - ab * pm.y, d.y, rd.y);
        const int o = w + k * wp;
        if (a0 && a1)
            O[o] = make_float2(v0, v1);
        else if (a0)
            pout[2 * o] = v0;
        else if (a1)
            pout[2 * o + 1] = v1;
        pm = pc;
        pc = pp;
        pp = pq;
        pS = sn;
        pN = nn;
        rc = rn;
        xw = xwn;
        xe = xen;
    }
    cp_async_wait<0>();  // (no copy outlives the block)
}

// Blocks of k_jacobi_pairs resident on the device at once (SMs x blocks per
// SM), set by jacobi_tb_configure.
static int jp_wave = 4 * 148;

// z chunk of the paired sweep: the longest chunk (fewest reloaded planes)
// whose launch fills its last wave of blocks to 85 % or more, else the one
// that fills it best (measured on a B200 at 200^3: 7 chunks of 29 planes in
// one wave, or 13 of 16 in 1.7 waves, 0.31 ms per 10 sweeps; 8 of 25 in 1.07
// waves 0.39 ms).  Down to one plane on small grids.  VOF_JACOBI_KCHUNK
// overrides.
static int jr_wave = 4 * 148;  // the same for k_jacobi_ring

int wave_kchunk(int nz, int bx, int wave) {
    int best = nz;
    double best_fill = -1.0;
    for (int n = 1; n <= nz; ++n) {
        const int kc = (nz + n - 1) / n;  // n chunks of (nearly) equal length
        const long long blocks = (long long)bx * ((nz + kc - 1) / kc);
        const long long waves = (blocks + wave - 1) / wave;
        const double fill = (double)blocks / (double)(waves * wave);
        if (fill >= 0.85) return kc;
        if (fill > best_fill) {
            best_fill = fill;
            best = kc;
        }
    }
    return best;
}

static int jacobi_pairs_kchunk(const Geom& g, int bx, int wave = jp_wave) {
    static int forced = -1;
    if (forced < 0) {
        const char* v = getenv("VOF_JACOBI_KCHUNK");
        forced = v ? atoi(v) : 0;
    }
    if (forced > 0) return forced < g.nz ? forced : g.nz;
    return wave_kchunk(g.nz, bx, wave);
}


cudaError_t jacobi_pairs_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s) {
    const int nq = (g.nx / 2 + 1) * g.ny;
    const int bx = (nq + JP_THREADS - 1) / JP_THREADS;
    const int kchunk = jacobi_pairs_kchunk(g, bx);
    k_jacobi_pairs<<<dim3(bx, (g.nz + kchunk - 1) / kchunk), JP_THREADS, 0, s>>>(g, pin, rhs, pout, kchunk);
    return cudaGetLastError();
}

static int jpe_wave = 3 * 148;  // resident blocks of the chosen k_jacobi_peel, set by jacobi_tb_configure
static int jq_wave = 3 * 148;   // the same for k_jacobi_quad

cudaError_t jacobi_quad_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s) {
    if (g.nx < 4) return jacobi_pairs_launch(g, pin, rhs, pout, s);  // two x-wall cells in one quad
    const int nq = (g.nx / 4 + 1) * g.ny;
    const int bx = (nq + 255) / 256;
    const int kchunk = jacobi_pairs_kchunk(g, bx, jq_wave);
    k_jacobi_quad<<<dim3(bx, (g.nz + kchunk - 1) / kchunk), 256, 0, s>>>(g, pin, rhs, pout, kchunk);
    return cudaGetLastError();
}

cudaError_t jacobi_peel_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s,
                               bool down) {
    const int nq = (g.nx / 2 + 1) * g.ny;
    const int bx = (nq + JP_THREADS - 1) / JP_THREADS;
    const int kchunk = jacobi_pairs_kchunk(g, bx, jpe_wave);
    const dim3 grid(bx, (g.nz + kchunk - 1) / kchunk);
    if (down)
        k_jacobi_peel<2, 4, true><<<grid, JP_THREADS, 0, s>>>(g, pin, rhs, pout, kchunk);
    else
        jp_peel_kernel()<<<grid, JP_THREADS, 0, s>>>(g, pin, rhs, pout, kchunk);
    return cudaGetLastError();
}

cudaError_t jacobi_ring_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s) {
    const int nq = (g.nx / 2 + 1) * g.ny;
    const int bx = (nq + JP_THREADS - 1) / JP_THREADS;
    const int kchunk = jacobi_pairs_kchunk(g, bx, jr_wave);
    k_jacobi_ring<<<dim3(bx, (g.nz + kchunk - 1) / kchunk), JP_THREADS, 0, s>>>(g, pin, rhs, pout, kchunk);
    return cudaGetLastError();
}

// Launch shape of k_jacobi_bulk: rows per block (BY * npair pairs must fit
// one block with its producer warp) and the z chunk from the resident-block
// count (the occupancy of that shape).  Cached for the last grid.
struct JSPlan {
    int nx, ny, nz, px;
    int by, slots, threads, kchunk, bx;
    size_t smem;
    bool ok;
};

static bool js_plan(const Geom& g, JSPlan* out) {
    static JSPlan last{};
    if (last.nx == g.nx && last.ny == g.ny && last.nz == g.nz && last.px == g.px && last.threads > 0) {
        *out = last;
        return last.ok;
    }
    JSPlan p{};
    p.nx = g.nx;
    p.ny = g.ny;
    p.nz = g.nz;
    p.px = g.px;
    const int npair = g.nx / 2 + 1;
    static int force_by = -1;
    if (force_by < 0) {
        const char* v = getenv("VOF_JS_BY");
        force_by = v ? atoi(v) : 0;
    }
    int by = (force_by == 1 || force_by == 2 || force_by == 4) ? force_by : 4;
    while (by > 1 && by * npair > 480) by >>= 1;
    p.ok = by * npair <= 480;
    const size_t bars = 2 * JS_SLOTS * sizeof(uint64_t);
    const size_t slot_bytes = (size_t)(2 * by + 2) * g.px * sizeof(float);
    const int slots = JS_SLOTS;
    p.smem = slots * slot_bytes + bars;
    p.ok = p.ok && p.smem <= (size_t)227 * 1024;
    p.by = by;
    p.slots = slots;
    p.threads = ((by * npair + 31) / 32) * 32 + 32;
    p.bx = (g.ny + by - 1) / by;
    int occ = 0, dev = 0, sms = 148;
    if (p.ok) {
        const void* k = by == 4 ? (const void*)k_jacobi_bulk<4> : by == 2 ? (const void*)k_jacobi_bulk<2>
                                                                          : (const void*)k_jacobi_bulk<1>;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, p.threads, p.smem) != cudaSuccess)
            occ = 0;
        p.ok = occ > 0;
    }
    p.kchunk = jacobi_pairs_kchunk(g, p.bx, (occ > 0 ? occ : 1) * sms);
    last = p;
    *out = p;
    return p.ok;
}

bool jacobi_bulk_supported(const Geom& g) {
    JSPlan p;
    return js_plan(g, &p);
}

cudaError_t jacobi_bulk_launch(const Geom& g, const float* pin, const float* rhs, float* pout, int* status,
                               cudaStream_t s) {
    JSPlan p;
    if (!js_plan(g, &p)) return cudaErrorInvalidValue;
    const dim3 grid(p.bx, (g.nz + p.kchunk - 1) / p.kchunk);
    switch (p.by) {
        case 4: k_jacobi_bulk<4><<<grid, p.threads, p.smem, s>>>(g, pin, rhs, pout, p.kchunk, status); break;
        case 2: k_jacobi_bulk<2><<<grid, p.threads, p.smem, s>>>(g, pin, rhs, pout, p.kchunk, status); break;
        default: k_jacobi_bulk<1><<<grid, p.threads, p.smem, s>>>(g, pin, rhs, pout, p.kchunk, status); break;
    }
    return cudaGetLastError();
}


// ---- two sweeps per launch, two cells per thread, marching z ----------------
// The pressure and rhs of a plane are read from memory once for two sweeps,
// so a pair of sweeps moves the bytes of one (read p, rhs; write p).
//
// A block owns a tile of `rows` rows by `tpx` pairs and a range of planes.
// Its threads cover the tile plus a one-row halo above and below (and, when
// a tile is narrower than a row, a one-pair halo left and right): the region
// of rh x rw pairs, numbered flat (pair fastest), one thread per pair.  At
// plane s a thread
//   - computes the first sweep of its pair at plane s from the input planes
//     s-1, s, s+1 of its own column (registers) and of its in-plane
//     neighbours (the input plane s in shared memory; the rows beyond the
//     region from memory),
//   - stores it in a ring of three first-sweep planes in shared memory,
//   - and, after the block's one barrier of the plane, computes the second
//     sweep of its pair (tile pairs only) at plane s-1 from the first-sweep
//     planes s-2, s-1, s of its own column (registers) and its neighbours'
//     plane s-1 (shared memory).
// The first sweep runs one plane beyond each end of the range.  Cells that
// are not updated (ghost rows, columns and planes) carry the input's value,
// as in k_jacobi_tb; they enter the second sweep only through zero
// coefficients.  Every update is the scalar expression of k_jacobi_pairs in
// the same operand order, so two sweeps here give the bits of two launches
// of that kernel.
//
// Work is dealt to a persistent grid (one block of up to 1024 threads per
// SM): the units are (tile, plane) with the plane fastest, and block b takes
// the contiguous units [b U / G, (b + 1) U / G), one segment per tile it
// touches, so every block marches the same number of planes.
struct J2Plan {
    int npair;     // pairs per row: columns 0 .. 2 npair - 1 cover 0 .. nx
    int tpx, ntx;  // pairs per tile along x, tiles along x
    int xh;        // halo pairs on each side along x (0: a tile is whole rows)
    int rows, nty; // rows per tile, tiles along y
    int rw, rh;    // region: pairs per row (tpx + 2 xh) and rows (rows + 2)
    long long units;
};

constexpr int J2_THREADS = 1024;

// Diagonals a_p = -(ae + aw + an + as + af + ab) (the reference's operand
// order) and their IEEE reciprocals for every pattern of wall sides: index
// (e*1 + w*2 + n*4 + s*8) * 4 + (bottom plane) + 2*(top plane), a bit set
// where that side's coefficient is the full one (the neighbour is not
// beyond a wall).  Built by the block's first 64 threads.
__device__ __forceinline__ void j2_diag_table(float2* tab, float cx, float cy, float cz) {
    const int e = threadIdx.x;
    if (e < 64) {
        const int pat = e >> 2, cls = e & 3;
        const float ae = (pat & 1) ? cx : 0.0f, aw = (pat & 2) ? cx : 0.0f;
        const float an = (pat & 4) ? cy : 0.0f, as = (pat & 8) ? cy : 0.0f;
        const float ab = (cls & 1) ? 0.0f : cz, af = (cls & 2) ? 0.0f : cz;
        const float d = -(ae + aw + an + as + af + ab);
        tab[e] = make_float2(d, __frcp_rn(d));
    }
}

__global__ void __launch_bounds__(J2_THREADS, 1) k_jacobi_pairs2(Geom g, const float* __restrict__ pin,
                                                               const float* __restrict__ rhs,
                                                               float* __restrict__ pout, J2Plan pl) {
    extern __shared__ float2 j2s[];
    const int RS = pl.rw * pl.rh;  // pairs of one region plane
    float2* s0 = j2s;              // [2][RS] input planes
    float2* s1 = j2s + 2 * RS;     // [3][RS] first-sweep planes
    float2* tab = j2s + 5 * RS;    // [64] diagonals (j2_diag_table)
    const int t = threadIdx.x;
    const bool tin = t < RS;
    const int lr = tin ? t / pl.rw : 0, lm = tin ? t - lr * pl.rw : 0;
    const float cx = g.dxi * g.dxi, cy = g.dyi * g.dyi, cz = g.dzi * g.dzi;
    j2_diag_table(tab, cx, cy, cz);
    const int wp = g.plane >> 1, wr = g.px >> 1;
    const float2* P = reinterpret_cast<const float2*>(pin);
    const float2* R = reinterpret_cast<const float2*>(rhs);
    float2* O = reinterpret_cast<float2*>(pout);
    const float2 zero = make_float2(0.0f, 0.0f);
    const long long G = gridDim.x;
    const long long ub = pl.units * blockIdx.x / G, ue = pl.units * (blockIdx.x + 1) / G;
    for (long long u = ub; u < ue;) {
        const int tile = (int)(u / g.nz);
        const long long tend = (long long)(tile + 1) * g.nz;
        const long long uend = ue < tend ? ue : tend;
        const int k0 = 1 + (int)(u - (long long)tile * g.nz), k1 = (int)(uend - (long long)tile * g.nz);
        u = uend;
        const int ty = tile / pl.ntx, tx = tile - ty * pl.ntx;
        const int j = ty * pl.rows + lr;  // region row 0 is the row before the tile's first
        const int m = tx * pl.tpx - pl.xh + lm;
        const bool valid = tin && j <= g.ny + 1 && m >= 0 && m < pl.npair;
        const int jc = valid ? j : 0, mc = valid ? m : 0;  // in-bounds addresses for every thread
        const int i0 = 2 * mc, i1 = i0 + 1;
        const bool rowin = valid && jc >= 1 && jc <= g.ny;
        const bool a0 = rowin && i0 >= 1, a1 = rowin && i1 <= g.nx;
        const bool out2 = rowin && lr >= 1 && lr <= pl.rows && lm >= pl.xh && lm < pl.xh + pl.tpx;
        const float ae0 = (i0 != g.nx) ? cx : 0.0f, aw0 = (i0 != 1) ? cx : 0.0f;
        const float ae1 = (i1 != g.nx) ? cx : 0.0f, aw1 = (i1 != 1) ? cx : 0.0f;
        const float an = (jc != g.ny) ? cy : 0.0f, as = (jc != 1) ? cy : 0.0f;
        const int pj = (jc != g.ny ? 4 : 0) | (jc != 1 ? 8 : 0);
        const int t0 = ((i0 != g.nx ? 1 : 0) | (i0 != 1 ? 2 : 0) | pj) * 4;
        const int t1 = ((i1 != g.nx ? 1 : 0) | (i1 != 1 ? 2 : 0) | pj) * 4;
        const int w = ((jc * g.px) >> 1) + mc;
        // the halo rows take their outer y neighbour from memory
        const bool lo_edge = lr == 0, hi_edge = lr == pl.rh - 1;
        const bool need_o = rowin && (lo_edge || hi_edge);
        const int wo = lo_edge ? w - wr : w + wr;
        const bool wpair = mc > 0 && lm > 0, epair = lm < pl.rw - 1;  // x neighbours inside the region
        const int sa = k0 - 1, sb = k1 + 1;
        float2 pm = P[w + (sa > 0 ? sa - 1 : 0) * wp], pc = P[w + sa * wp], pp = P[w + (sa + 1) * wp];
        float2 po = need_o ? P[wo + sa * wp] : zero;
        float2 rc = R[w + sa * wp], r1 = zero;
        float2 qm = zero, qc = zero, qp = zero;  // first-sweep values at s-2, s-1, s
        if (tin) s0[(sa & 1) * RS + t] = pc;
        __syncthreads();
        int s3 = sa % 3;  // s % 3
        for (int s = sa; s <= sb; ++s) {
            const bool more = s < sb;
            const int s2 = s + 2 > g.nz + 1 ? g.nz + 1 : s + 2;
            const float2 pq = more ? P[w + s2 * wp] : zero;
            const float2 pon = (more && need_o) ? P[wo + (s + 1) * wp] : zero;
            const float2 rn = more ? R[w + (s + 1) * wp] : zero;
            // first sweep at plane s
            float2 v = pc;
            if (rowin && s >= 1 && s <= g.nz) {
                const float2* S0 = s0 + (s & 1) * RS + t;
                const float pw = wpair ? S0[-1].y : 0.0f;
                const float pe = epair ? S0[1].x : 0.0f;
                const float2 pS = lo_edge ? po : S0[-pl.rw];
                const float2 pN = hi_edge ? po : S0[pl.rw];
                const bool kb = s == 1, kt = s == g.nz;
                const float af = kt ? 0.0f : cz, ab = kb ? 0.0f : cz;
                const int cls = (kb ? 1 : 0) | (kt ? 2 : 0);
                const float2 d0 = tab[t0 + cls], d1 = tab[t1 + cls];
                if (a0)
                    v.x = div_rn_pre(rc.x - ae0 * pc.y - aw0 * pw - an * pN.x - as * pS.x - af * pp.x - ab * pm.x,
                                     d0.x, d0.y);
                if (a1)
                    v.y = div_rn_pre(rc.y - ae1 * pe - aw1 * pc.x - an * pN.y - as * pS.y - af * pp.y - ab * pm.y,
                                     d1.x, d1.y);
            }
            qm = qc;
            qc = qp;
            qp = v;
            if (tin) {
                s1[s3 * RS + t] = v;
                if (more) s0[((s + 1) & 1) * RS + t] = pp;
            }
            __syncthreads();
            // second sweep at plane s - 1
            const int q = s - 1;
            if (q >= k0 && out2) {
                const float2* S1 = s1 + (s3 == 0 ? 2 : s3 - 1) * RS + t;
                const float pw = mc > 0 ? S1[-1].y : 0.0f;
                const float pe = epair ? S1[1].x : 0.0f;
                const float2 pS = S1[-pl.rw], pN = S1[pl.rw];
                const bool kb = q == 1, kt = q == g.nz;
                const float af = kt ? 0.0f : cz, ab = kb ? 0.0f : cz;
                const int cls = (kb ? 1 : 0) | (kt ? 2 : 0);
                const float2 d0 = tab[t0 + cls], d1 = tab[t1 + cls];
                const float v0 =
                    div_rn_pre(r1.x - ae0 * qc.y - aw0 * pw - an * pN.x - as * pS.x - af * qp.x - ab * qm.x, d0.x,
                               d0.y);
                const float v1 =
                    div_rn_pre(r1.y - ae1 * pe - aw1 * qc.x - an * pN.y - as * pS.y - af * qp.y - ab * qm.y, d1.x,
                               d1.y);
                const int o = w + q * wp;
                if (a0 && a1)
                    O[o] = make_float2(v0, v1);
                else if (a0)
                    pout[2 * o] = v0;
                else if (a1)
                    pout[2 * o + 1] = v1;
            }
            r1 = rc;
            rc = rn;
            pm = pc;
            pc = pp;
            pp = pq;
            po = pon;
            s3 = s3 == 2 ? 0 : s3 + 1;
        }
        __syncthreads();  // the next segment reuses the planes
    }
}

static int j2_blocks = 148;  // resident blocks of k_jacobi_pairs2 (SMs x 1), set by jacobi_tb_configure

// Tile shape: for 1, 2, 3 ... tiles along x, the widest region that fits a
// block (at least four tile rows), keeping the shape with the least
// first-sweep work per output pair.
static J2Plan j2_plan(const Geom& g) {
    J2Plan best{};
    double best_cost = 1e300;
    const int npair = g.nx / 2 + 1;
    for (int ntx = 1; ntx <= 64; ++ntx) {
        J2Plan p{};
        p.npair = npair;
        p.ntx = ntx;
        p.tpx = (npair + ntx - 1) / ntx;
        if (ntx > 1 && (p.tpx - 1) * ntx >= npair) continue;  // same tiles as fewer of them
        p.xh = ntx > 1 ? 1 : 0;
        p.rw = p.tpx + 2 * p.xh;
        if (p.rw > J2_THREADS / 6) continue;
        p.rh = J2_THREADS / p.rw;
        p.rows = p.rh - 2;
        if (p.rows > g.ny) {
            p.rows = g.ny;
            p.rh = p.rows + 2;
        }
        p.nty = (g.ny + p.rows - 1) / p.rows;
        p.units = (long long)p.ntx * p.nty * g.nz;
        const double cost = (double)p.rw * p.rh / ((double)p.tpx * p.rows);
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = p;
        }
    }
    return best;
}

bool jacobi_pairs2_supported(const Geom& g) {
    const J2Plan p = j2_plan(g);
    return p.rw > 0 && p.rows >= 1 && g.px % 2 == 0;
}

cudaError_t jacobi_pairs2_launch(const Geom& g, const float* pin, const float* rhs, float* pout, cudaStream_t s) {
    const J2Plan p = j2_plan(g);
    if (p.rw <= 0) return cudaErrorInvalidValue;
    // at least about four planes per block: shorter ranges spend most of
    // their time on the extra first-sweep planes at their ends
    long long nb = p.units / 4;
    if (nb > j2_blocks) nb = j2_blocks;
    if (nb < 1) nb = 1;
    const size_t smem = sizeof(float2) * (5u * (size_t)p.rw * p.rh + 64u);
    k_jacobi_pairs2<<<(unsigned)nb, J2_THREADS, smem, s>>>(g, pin, rhs, pout, p);
    return cudaGetLastError();
}

size_t jacobi_tb_smem_bytes(int T) {
    switch (T) {
        case 1: return JTile<1>::SMEM;
        case 2: return JTile<2>::SMEM;
        case 3: return JTile<3>::SMEM;
        case 4: return JTile<4>::SMEM;
        default: return 0;
    }
}

cudaError_t jacobi_tb_configure() {
    cudaError_t e;
    int dev = 0, sms = 0, occ = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_jacobi_pairs, JP_THREADS, 0)) != cudaSuccess)
        return e;
    jp_wave = (sms > 0 ? sms : 148) * (occ > 0 ? occ : 1);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_jacobi_ring, JP_THREADS, 0)) != cudaSuccess)
        return e;
    jr_wave = (sms > 0 ? sms : 148) * (occ > 0 ? occ : 1);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, jp_peel_kernel(), JP_THREADS, 0)) != cudaSuccess)
        return e;
    jpe_wave = (sms > 0 ? sms : 148) * (occ > 0 ? occ : 1);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_jacobi_quad, 256, 0)) != cudaSuccess) return e;
    jq_wave = (sms > 0 ? sms : 148) * (occ > 0 ? occ : 1);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_jacobi_pairs2, J2_THREADS,
                                                           sizeof(float2) * (5u * J2_THREADS + 64u))) != cudaSuccess)
        return e;
    j2_blocks = (sms > 0 ? sms : 148) * (occ > 0 ? occ : 1);
    for (const void* k : {(const void*)k_jacobi_bulk<4>, (const void*)k_jacobi_bulk<2>, (const void*)k_jacobi_bulk<1>})
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
            return e;
    if ((e = cudaFuncSetAttribute(k_jacobi_bulk<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024)) !=
            cudaSuccess ||
        (e = cudaFuncSetAttribute(k_jacobi_bulk<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024)) !=
            cudaSuccess ||
        (e = cudaFuncSetAttribute(k_jacobi_bulk<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024)) !=
            cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_jacobi_tb<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)JTile<1>::SMEM)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_jacobi_tb<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)JTile<2>::SMEM)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_jacobi_tb<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)JTile<3>::SMEM)) != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(k_jacobi_tb<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)JTile<4>::SMEM);
}

cudaError_t jacobi_tb_maps(const Geom& g, const float* field, CUtensorMap* map) {
    return make_tensor_map_3d(map, field, g.px, g.py, g.nz + 2, JB_W, JB_EY, 1);
}

template <int T>
static dim3 tb_grid(const Geom& g, int kchunk) {
    return dim3((g.nx + JTile<T>::BX - 1) / JTile<T>::BX, (g.ny + JTile<T>::BY - 1) / JTile<T>::BY,
                (g.nz + kchunk - 1) / kchunk);
}

cudaError_t jacobi_tb_launch(const Geom& g, int T, const CUtensorMap& map_in, const CUtensorMap& map_rhs,
                             float* pout, int* status, cudaStream_t s) {
    // z chunks long enough that the T-plane warm-up at each end is small,
    // and enough blocks to fill the GPU for a few waves.  On small grids the
    // chunks shrink (down to one plane) until the launch has about 600
    // blocks: a few blocks marching 16 planes each are bound by the latency
    // of their plane pipeline.
    const long long tiles = (long long)((g.nx + JB_TX - 1) / JB_TX + 1) * ((g.ny + JB_TX - 1) / JB_TX + 1);
    const int target = (int)((long long)g.nz * tiles / 600);
    const int kchunk = target < 1 ? 1 : (target > 16 ? 16 : target);
    const dim3 blk(JB_TX, JB_TY);
    switch (T) {
        case 1: k_jacobi_tb<1><<<tb_grid<1>(g, kchunk), blk, JTile<1>::SMEM, s>>>(g, map_in, map_rhs, pout, kchunk, status); break;
        case 2: k_jacobi_tb<2><<<tb_grid<2>(g, kchunk), blk, JTile<2>::SMEM, s>>>(g, map_in, map_rhs, pout, kchunk, status); break;
        case 3: k_jacobi_tb<3><<<tb_grid<3>(g, kchunk), blk, JTile<3>::SMEM, s>>>(g, map_in, map_rhs, pout, kchunk, status); break;
        case 4: k_jacobi_tb<4><<<tb_grid<4>(g, kchunk), blk, JTile<4>::SMEM, s>>>(g, map_in, map_rhs, pout, kchunk, status); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace vof
