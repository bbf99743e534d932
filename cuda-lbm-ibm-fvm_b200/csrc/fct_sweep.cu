// fct_sweep.cu -- one directionally split FCT sweep of the volume fraction
// (fct_{x,y,z}_sweep_stage1..4, voftrial1.cu:509-905) as a single kernel.
//
// Compiled with -fmad=false like plain_step.cu: every expression below keeps
// the reference's operand order and no multiply-add is contracted.
//
// Why the four reference stages collapse into one pass over a grid line.
// Stage 2 of a sweep zeroes the other direction's antidiffusive fluxes
// (voftrial1.cu:573-574, 712-713), so the terms they contribute to pp, pm and
// the stage-4 update vanish (exactly, up to the sign of a zero, which the
// final clamp01f removes).  What is left couples only cells of the same line
// along the sweep axis, with a reach of three cells.  The zero-filled buffers
// the reference never writes (voftrial1.cu:1200-1203) fix the line ends:
//   Ftd at the two ghost cells is 0, rp and rm at the ghost cells are 0, and
//   the limiter c of the first face (c[1]) is 0; the wall-face velocities
//   are 0 after apply_bc_velocity, so the ghost F values enter only as 0*F.
//
// The per-cell expressions (and the reference's length factors per sweep)
// are in fct_line.cuh, shared with the sweep adjoint.
//
// Kernel shape.  A block owns a tile of 32 lines (one per lane; lines are
// numbered over both cross axes) over their full length.  The tile's F and
// face velocity are staged once in shared memory with coalesced loads; then
// each warp marches one segment of the
// lines, carrying the stage values of the last few cells in registers, so each
// cell's fluxes, Ftd, Zalesak ratios and face limiters are computed exactly
// once (plus a three-cell warm-up at segment starts).  Shared memory is laid
// out so a warp's 32 lanes (32 lines, same position) hit 32 banks:
//   x lines: [line][pos] with an odd row pitch;  y/z lines: [pos][line].
// y/z lines are contiguous across lanes in HBM, so results go straight to
// global memory; x results are staged in the F tile and written back row-wise.
#include <cuda_runtime.h>

#include "fct_line.cuh"
#include "fct_sweep.h"

namespace vof {

#if defined(__CUDA_ARCH__) && !defined(VOF_FMAD_FALSE)
#error "fct_sweep.cu must be compiled with -fmad=false -DVOF_FMAD_FALSE"
#endif

namespace {

constexpr int LANES = 32;     // lines per tile
constexpr int WARPS = 8;      // segments per line
constexpr int THREADS = LANES * WARPS;

__host__ __device__ inline int odd_pitch(int npos) { return npos | 1; }

using fct::Sweep;
using fct::face_limit;
using fct::ftd_from;
using fct::limiter;

// Line accessor: smem values of one lane's line at position q.
struct LineView {
    const float* f;
    const float* v;
    int qs;  // smem stride between consecutive positions
    __device__ __forceinline__ float F(int q) const { return f[q * qs]; }
    __device__ __forceinline__ float V(int q) const { return v[q * qs]; }
};

// Low-order flux and antidiffusive flux through face fidx (between cells
// fidx-1 and fidx), as fl_L / fl_H of the reference's stages 1-2.
__device__ __forceinline__ void face_flux(const LineView& L, int fidx, float dt, float& lo, float& a) {
    fct::flux(L.V(fidx), L.F(fidx - 1), L.F(fidx), dt, lo, a);
}

template <int AXIS>
__device__ __forceinline__ float cell_dv(const Sweep<AXIS>& S, const LineView& L, int c) {
    return S.dv(L.V(c), L.V(c + 1));
}

// ---- from-scratch evaluation (segment warm-up only) -------------------------
template <int AXIS>
__device__ float ftd_at(const Sweep<AXIS>& S, const Geom& g, const LineView& L, int c) {
    if (c < 1 || c > S.n) return 0.0f;
    float lo_in, lo_out, a;
    face_flux(L, c, S.dt, lo_in, a);
    face_flux(L, c + 1, S.dt, lo_out, a);
    const float dv = cell_dv(S, L, c);
    return ftd_from(S, L.F(c), lo_in, lo_out, dv, __frcp_rn(dv));
}

__device__ __forceinline__ float a_at(const LineView& L, int f, int n, float dt) {
    if (f < 1 || f > n + 1) return 0.0f;
    float lo, a;
    face_flux(L, f, dt, lo, a);
    return a;
}

template <int AXIS>
__device__ void ratios_at(const Sweep<AXIS>& S, const Geom& g, const LineView& L, int c, float& rp, float& rm) {
    if (c < 1 || c > S.n) {
        rp = 0.0f;
        rm = 0.0f;
        return;
    }
    limiter(S, ftd_at(S, g, L, c - 1), ftd_at(S, g, L, c), ftd_at(S, g, L, c + 1), a_at(L, c, S.n, S.dt),
            a_at(L, c + 1, S.n, S.dt), rp, rm);
}

// Indices whose clamped value is x on an axis of n interior cells: x itself,
// plus the ghost 0 when x == 1 and the ghost n+1 when x == n.
__device__ __forceinline__ int mirrors(int x, int n, int* out) {
    out[0] = x;  // fixed positions (no runtime index)
    out[1] = (x == 1) ? 0 : n + 1;
    out[2] = n + 1;
    return 1 + (x == 1) + (x == n);
}

// apply_bc_F (voftrial1.cu:1122-1135) for one cell of the final sweep: the
// cell (i, j, k) and every ghost whose clamped interior index is (i, j, k)
// take f.  Out of line: only cells on the domain's edge come here, and inlined
// it would hold registers in every thread of the marching kernels.
__device__ __noinline__ void store_mirrored(float* __restrict__ F, int px, int plane, int nx, int ny, int nz, int i,
                                            int j, int k, float f) {
    int iv[3], jv[3], kv[3];
    const int ni = mirrors(i, nx, iv), nj = mirrors(j, ny, jv), nk = mirrors(k, nz, kv);
    for (int c = 0; c < nk; ++c)
        for (int b = 0; b < nj; ++b)
            for (int a = 0; a < ni; ++a) F[kv[c] * plane + jv[b] * px + iv[a]] = f;
}

}  // namespace

// ---- one tile ---------------------------------------------------------------
template <int AXIS, bool FINAL>
// Fsrc: the sweep's input F (staged into shared memory first); F: its output
// (interior cells, and on the final sweep every ghost cell).  They may be the
// same buffer (in place); otherwise F's ghost cells must hold finite values
// on a non-final sweep (the next sweep reads them only through wall-face
// fluxes of zero velocity).
__global__ void __launch_bounds__(THREADS, 2) k_fct(Geom g, const float* Fsrc, float* F,
                                                    const float* __restrict__ vel) {
    extern __shared__ float smem[];
    const Sweep<AXIS> S(g);
    const int n = S.n;
    const int npos = n + 2;
    const int na = AXIS == 0 ? g.ny : g.nx;           // lines along a
    const int nb = AXIS == 2 ? g.ny : g.nz;           // lines along b
    const int lane = threadIdx.x, warp = threadIdx.y;
    // the tile's lines (a, b), numbered a fastest over both cross axes so
    // that no lane idles at the end of a row of lines
    const int line0 = blockIdx.x * LANES;             // first line of the tile
    const int nl = min(LANES, na * nb - line0);
    auto line_a = [&](int l) { return 1 + (line0 + l) % na; };
    auto line_b = [&](int l) { return 1 + (line0 + l) / na; };
    const int P = odd_pitch(npos);

    // global index of (line a, b; position q)
    auto gi = [&](int a, int bb, int q) {
        return AXIS == 0 ? gidx(g, q, a, bb) : (AXIS == 1 ? gidx(g, a, q, bb) : gidx(g, a, bb, q));
    };
    // shared index of (line l, position q)
    const int qs = AXIS == 0 ? 1 : LANES;
    auto si = [&](int l, int q) { return AXIS == 0 ? l * P + q : q * LANES + l; };
    const int tile = AXIS == 0 ? LANES * P : npos * LANES;
    float* sF = smem;  // x lines: also the staged results, written in place (below)
    float* sV = smem + tile;

    // ---- stage the tile (coalesced) ----
    if (AXIS == 0) {
        for (int l = warp; l < nl; l += WARPS) {
            const int base = gi(line_a(l), line_b(l), 0);
            for (int q = lane; q < npos; q += LANES) {
                sF[l * P + q] = Fsrc[base + q];
                sV[l * P + q] = __ldg(vel + base + q);
            }
        }
    } else {
        if (lane < nl) {
            for (int q = warp; q < npos; q += WARPS) {
                const int gq = gi(line_a(lane), line_b(lane), q);
                sF[q * LANES + lane] = Fsrc[gq];
                sV[q * LANES + lane] = __ldg(vel + gq);
            }
        }
    }
    __syncthreads();

    // ---- march one segment of this lane's line ----
    const int seg = (n + WARPS - 1) / WARPS;
    const int c0 = 1 + warp * seg;
    const int c1 = min(n, c0 + seg - 1);
    const LineView L{sF + si(lane, 0), sV + si(lane, 0), qs};
    const int a = line_a(lane), b = line_b(lane);
    const bool live = lane < nl && c0 <= n;

    // x lines: each result goes into sF in place.  The march at cell c reads
    // F only at c+2 and c+3, so a warp never reads a cell it has written; the
    // warm-up below reads the three cells before the segment (the previous
    // warp's last cells), and the march reads the three after it (the next
    // warp's first cells): hence a barrier after the warm-ups, and each warp
    // holds its first three results in registers until every march is done.
    const float dt = S.dt;
    float lo2 = 0.0f, a0f = 0.0f, a1f = 0.0f, a2f = 0.0f, T0 = 0.0f, T1 = 0.0f, rp0 = 0.0f, rm0 = 0.0f;
    float cf0 = 0.0f, dv0 = 1.0f, dv1 = 1.0f, rdv0 = 1.0f, rdv1 = 1.0f;
    float held0 = 0.0f, held1 = 0.0f, held2 = 0.0f;
    if (live) {
        // state before cell c0
        {
            float lo_tmp;
            face_flux(L, c0, dt, lo_tmp, a0f);
            a1f = a_at(L, c0 + 1, n, dt);
            a2f = a_at(L, c0 + 2, n, dt);
            lo2 = 0.0f;
            if (c0 + 2 <= n + 1) face_flux(L, c0 + 2, dt, lo2, a2f);
            T0 = ftd_at(S, g, L, c0);
            T1 = ftd_at(S, g, L, c0 + 1);
            ratios_at(S, g, L, c0, rp0, rm0);
            if (c0 == 1) {
                cf0 = 0.0f;  // c[imin] is never written
            } else {
                float rpm, rmm;
                ratios_at(S, g, L, c0 - 1, rpm, rmm);
                cf0 = face_limit(a0f, rpm, rmm, rp0, rm0);
            }
            dv0 = cell_dv(S, L, c0);
            dv1 = (c0 + 1 <= n) ? cell_dv(S, L, c0 + 1) : 1.0f;
            rdv0 = __frcp_rn(dv0);
            rdv1 = __frcp_rn(dv1);
        }
    }
    if (AXIS == 0) __syncthreads();
    if (live) {
        for (int c = c0; c <= c1; ++c) {
            // face c+3, Ftd(c+2), ratios(c+1), limiter of face c+1, result of cell c
            float lo3 = 0.0f, a3f = 0.0f;
            if (c + 3 <= n + 1) face_flux(L, c + 3, dt, lo3, a3f);
            float T2 = 0.0f, dv2 = 1.0f, rdv2 = 1.0f;
            if (c + 2 <= n) {
                dv2 = cell_dv(S, L, c + 2);
                rdv2 = __frcp_rn(dv2);
                T2 = ftd_from(S, L.F(c + 2), lo2, lo3, dv2, rdv2);
            }
            float rp1 = 0.0f, rm1 = 0.0f;
            if (c + 1 <= n) limiter(S, T0, T1, T2, a1f, a2f, rp1, rm1);
            const float cf1 = face_limit(a1f, rp0, rm0, rp1, rm1);
            float fnew = clamp01f(fct::stage4(S, T0, a0f, cf0, a1f, cf1, dv0, rdv0));
            if (FINAL) fnew = clamp01f(fnew);  // post_process_f_kernel, voftrial1.cu:502-507

            if (AXIS == 0) {
                if (c == c0) held0 = fnew;
                else if (c == c0 + 1) held1 = fnew;
                else if (c == c0 + 2) held2 = fnew;
                else sF[lane * P + c] = fnew;
            } else if (!FINAL) {
                F[gi(a, b, c)] = fnew;
            } else {
                // apply_bc_F (voftrial1.cu:1122-1135) composes to: every ghost
                // cell takes the value at its clamped interior index.  Write the
                // interior cell and every ghost that maps onto it.
                int qv[3], av[3], bv[3];
                const int nq = mirrors(c, n, qv), nav = mirrors(a, na, av), nbv = mirrors(b, nb, bv);
                for (int ib = 0; ib < nbv; ++ib)
                    for (int ia = 0; ia < nav; ++ia)
                        for (int iq = 0; iq < nq; ++iq) F[gi(av[ia], bv[ib], qv[iq])] = fnew;
            }

            lo2 = lo3;
            a0f = a1f;
            a1f = a2f;
            a2f = a3f;
            T0 = T1;
            T1 = T2;
            rp0 = rp1;
            rm0 = rm1;
            cf0 = cf1;
            dv0 = dv1;
            dv1 = dv2;
            rdv0 = rdv1;
            rdv1 = rdv2;
        }
    }

    if (AXIS == 0) {
        __syncthreads();  // every march is done: the held results go in
        if (live) {
            sF[lane * P + c0] = held0;
            if (c0 + 1 <= c1) sF[lane * P + c0 + 1] = held1;
            if (c0 + 2 <= c1) sF[lane * P + c0 + 2] = held2;
        }
        // ---- write the x rows back (coalesced) ----
        __syncthreads();
        for (int l = warp; l < nl; l += WARPS) {
            const int aa = line_a(l), bb = line_b(l);
            if (!FINAL) {
                const int base = gi(aa, bb, 0);
                for (int q = 1 + lane; q <= n; q += LANES) F[base + q] = sF[l * P + q];
            } else {
                int av[3], bv[3];
                const int nav = mirrors(aa, na, av), nbv = mirrors(bb, nb, bv);
                for (int ib = 0; ib < nbv; ++ib)
                    for (int ia = 0; ia < nav; ++ia) {
                        const int base = gi(av[ia], bv[ib], 0);
                        for (int q = lane; q <= n + 1; q += LANES)
                            F[base + q] = sF[l * P + (q < 1 ? 1 : (q > n ? n : q))];
                    }
            }
        }
    }
}

// ---- y and z sweeps out of place: one thread per line segment ------------------
// Lines along y or z are contiguous across the 32 lanes of a warp (lanes run
// along x), so a lane reads its line's F and face velocity straight from
// memory, one coalesced row per position, with the next position's operands
// loaded an iteration ahead; no shared memory and no barrier.  The march and
// its register window are those of k_fct; the state before the segment's
// first cell comes from the Ftd of the four cells before it and the two
// ratios it needs.  Fin and Fout must be different buffers: a segment's
// warm-up reads the cells of the segment before it.
struct GLine {
    const float* f;
    const float* v;
    int qs;
    __device__ __forceinline__ float F(int q) const { return __ldg(f + (ptrdiff_t)q * qs); }
    __device__ __forceinline__ float V(int q) const { return __ldg(v + (ptrdiff_t)q * qs); }
};

template <int AXIS>
__device__ __forceinline__ float gftd(const Sweep<AXIS>& S, const GLine& L, int c) {
    if (c < 1 || c > S.n) return 0.0f;
    float lo_in, lo_out, a;
    fct::flux(L.V(c), L.F(c - 1), L.F(c), S.dt, lo_in, a);
    fct::flux(L.V(c + 1), L.F(c), L.F(c + 1), S.dt, lo_out, a);
    const float dv = S.dv(L.V(c), L.V(c + 1));
    return ftd_from(S, L.F(c), lo_in, lo_out, dv, __frcp_rn(dv));
}

__device__ __forceinline__ float ga(const GLine& L, int f, int n, float dt) {
    if (f < 1 || f > n + 1) return 0.0f;
    float lo, a;
    fct::flux(L.V(f), L.F(f - 1), L.F(f), dt, lo, a);
    return a;
}

constexpr int MARCH_THREADS = 256;
// Positions the march loads ahead of the one it uses, and its unroll factor
// (measured on a B200 at 200^3: two ahead, unrolled twice, the fastest of
// one or two ahead and one or two unrolled).
#ifndef VOF_MARCH_AHEAD
#define VOF_MARCH_AHEAD 2
#endif
#ifndef VOF_MARCH_UNROLL
#define VOF_MARCH_UNROLL 2
#endif

// Lines are numbered flat, i fastest (a warp may span two rows of lines:
// two coalesced pieces per load), blockIdx.y is the segment.
template <int AXIS, bool FINAL>
__global__ void __launch_bounds__(MARCH_THREADS, 4) k_fct_march(Geom g, const float* __restrict__ Fin,
                                                                float* __restrict__ F,
                                                                const float* __restrict__ vel, int seg) {
    static_assert(AXIS == 1 || AXIS == 2, "lines along y or z");
    const Sweep<AXIS> S(g);
    const int n = S.n;
    const int nb = AXIS == 1 ? g.nz : g.ny;
    const int line = blockIdx.x * MARCH_THREADS + threadIdx.x;
    const int a = 1 + line % g.nx;  // i
    const int b = 1 + line / g.nx;  // k (y lines) or j (z lines)
    const int c0 = 1 + blockIdx.y * seg;
    if (b > nb || c0 > n) return;
    const int c1 = min(n, c0 + seg - 1);
    auto gi = [&](int aa, int bb, int q) { return AXIS == 1 ? gidx(g, aa, q, bb) : gidx(g, aa, bb, q); };
    const int qs = AXIS == 1 ? g.px : g.plane;
    const int base = gi(a, b, 0);
    const GLine L{Fin + base, vel + base, qs};
    const float dt = S.dt;

    // state before cell c0 (as k_fct's march carries it into c0)
    float a0f, a1f, a2f, lo2 = 0.0f;
    {
        float lo_tmp;
        fct::flux(L.V(c0), L.F(c0 - 1), L.F(c0), dt, lo_tmp, a0f);
    }
    a1f = ga(L, c0 + 1, n, dt);
    a2f = 0.0f;
    if (c0 + 2 <= n + 1) fct::flux(L.V(c0 + 2), L.F(c0 + 1), L.F(c0 + 2), dt, lo2, a2f);
    const float Tm2 = gftd(S, L, c0 - 2), Tm1 = gftd(S, L, c0 - 1);
    float T0 = gftd(S, L, c0), T1 = gftd(S, L, c0 + 1);
    float rp0 = 0.0f, rm0 = 0.0f;
    limiter(S, Tm1, T0, T1, a0f, a1f, rp0, rm0);  // c0 is interior
    float cf0 = 0.0f;                             // c[1] is never written
    if (c0 > 1) {
        float rpm, rmm;
        limiter(S, Tm2, Tm1, T0, ga(L, c0 - 1, n, dt), a0f, rpm, rmm);
        cf0 = face_limit(a0f, rpm, rmm, rp0, rm0);
    }
    float dv0 = S.dv(L.V(c0), L.V(c0 + 1));
    float dv1 = (c0 + 1 <= n) ? S.dv(L.V(c0 + 1), L.V(c0 + 2)) : 1.0f;
    // operands of position c+3 for the first iteration, and a window of F/V
    float F2 = L.F(c0 + 2 <= n + 1 ? c0 + 2 : n + 1);
    float V3 = (c0 + 3 <= n + 1) ? L.V(c0 + 3) : 0.0f, F3 = (c0 + 3 <= n + 1) ? L.F(c0 + 3) : 0.0f;
    float V2 = (c0 + 2 <= n + 1) ? L.V(c0 + 2) : 0.0f;
    const int nm = AXIS == 1 ? g.ny : g.nz;
    // Run of positions, up to c+2 here and c+3 in the loop, where F is 0 and
    // |face velocity| < vq (positions off the line count as such).  vq keeps
    // every cell's dv = vol - dvfac (v_hi - v_lo) above 0.01 vol: finite and
    // positive, so a zero numerator gives a zero quotient.
    const float vq = 0.49f * S.vol / S.dvfac;
    int zrun = 0;
    for (int q = c0 - 3; q <= c0 + 2; ++q) {
        const bool in = q >= 0 && q <= n + 1;
        zrun = (!in || (L.F(q) == 0.0f && fabsf(L.V(q)) < vq)) ? zrun + 1 : 0;
    }
    // Final sweep, apply_bc_F (voftrial1.cu:1122-1135): every ghost takes the
    // value at its clamped interior index.  Across the line, a cell at a = 1
    // or nx, b = 1 or nb has ghost copies on those sides (and their corner),
    // written inline by the lines at the box's edge; the line's own ghosts
    // (c = 0 and n + 1, with their copies across) are written after the march
    // from the values kept at c = 1 and c = n.  No call inside the loop.
    const int bs = AXIS == 1 ? g.plane : g.px;  // b's stride
    const bool edge = a == 1 || a == g.nx || b == 1 || b == nb;
    float f_lo = 0.0f, f_hi = 0.0f;
#if VOF_MARCH_AHEAD >= 2
    float F4 = (c0 + 4 <= n + 1) ? L.F(c0 + 4) : 0.0f, V4 = (c0 + 4 <= n + 1) ? L.V(c0 + 4) : 0.0f;
#endif
    VOF_UNROLL(VOF_MARCH_UNROLL)
    for (int c = c0; c <= c1; ++c) {
#if VOF_MARCH_AHEAD >= 2
        // operands of position c+5, loaded two march steps ahead
        const bool nx5 = c + 5 <= n + 1 && c + 1 < c1;
        const float V5 = nx5 ? L.V(c + 5) : 0.0f, F5 = nx5 ? L.F(c + 5) : 0.0f;
#else
        // next iteration's operands (position c+4), loaded a march step ahead
        const bool nx4 = c + 4 <= n + 1 && c < c1;
        const float V4 = nx4 ? L.V(c + 4) : 0.0f, F4 = nx4 ? L.F(c + 4) : 0.0f;
#endif
        // F == 0 at positions c-3 .. c+3 (velocities below vq): every stage
        // value this iteration forms -- the flux of face c+3, Ftd(c+2), the
        // ratios of c+1, the limiter of face c+1 and the new F(c) -- is zero
        // (up to the sign of a zero, which no comparison sees and the final
        // clamp01f removes), and so is the carried window.  Only dv(c+2) is
        // needed later.  Most of a dam break is gas, far from the interface.
        zrun = (F3 == 0.0f && fabsf(V3) < vq) ? zrun + 1 : 0;
        const bool quiet = zrun >= 7;
        const float dv2 = (c + 2 <= n) ? S.dv(V2, V3) : 1.0f;
        float lo3 = 0.0f, a3f = 0.0f, T2 = 0.0f, rp1 = 0.0f, rm1 = 0.0f, cf1 = 0.0f, fnew = 0.0f;
        if (!quiet) {
            if (c + 3 <= n + 1) fct::flux(V3, F2, F3, dt, lo3, a3f);
            if (c + 2 <= n) T2 = ftd_from(S, F2, lo2, lo3, dv2, __frcp_rn(dv2));
            if (c + 1 <= n) limiter(S, T0, T1, T2, a1f, a2f, rp1, rm1);
            cf1 = face_limit(a1f, rp0, rm0, rp1, rm1);
            // (the reciprocal of dv(c) formed again here rather than carried:
            // quiet positions skip it)
            fnew = clamp01f(fct::stage4(S, T0, a0f, cf0, a1f, cf1, dv0, __frcp_rn(dv0)));
        }
        if (!FINAL) {
            F[gi(a, b, c)] = fnew;
        } else {
            fnew = clamp01f(fnew);  // post_process_f_kernel, voftrial1.cu:502-507
            const int o = gi(a, b, c);
            F[o] = fnew;
            if (edge) {
                if (a == 1) F[o - 1] = fnew;
                if (a == g.nx) F[o + 1] = fnew;
                if (b == 1) {
                    F[o - bs] = fnew;
                    if (a == 1) F[o - bs - 1] = fnew;
                    if (a == g.nx) F[o - bs + 1] = fnew;
                }
                if (b == nb) {
                    F[o + bs] = fnew;
                    if (a == 1) F[o + bs - 1] = fnew;
                    if (a == g.nx) F[o + bs + 1] = fnew;
                }
            }
            if (c == 1) f_lo = fnew;
            if (c == nm) f_hi = fnew;
        }
        lo2 = lo3;
        a0f = a1f;
        a1f = a2f;
        a2f = a3f;
        T0 = T1;
        T1 = T2;
        rp0 = rp1;
        rm0 = rm1;
        cf0 = cf1;
        dv0 = dv1;
        dv1 = dv2;
        F2 = F3;
        F3 = F4;
        V2 = V3;
        V3 = V4;
#if VOF_MARCH_AHEAD >= 2
        F4 = F5;
        V4 = V5;
#endif
    }
    if (FINAL) {
        if (AXIS == 1) {  // (a, b, c) = (i, k, j)
            if (c0 == 1) store_mirrored(F, g.px, g.plane, g.nx, g.ny, g.nz, a, 1, b, f_lo);
            if (c1 == nm) store_mirrored(F, g.px, g.plane, g.nx, g.ny, g.nz, a, nm, b, f_hi);
        } else {  // (a, b, c) = (i, j, k)
            if (c0 == 1) store_mirrored(F, g.px, g.plane, g.nx, g.ny, g.nz, a, b, 1, f_lo);
            if (c1 == nm) store_mirrored(F, g.px, g.plane, g.nx, g.ny, g.nz, a, b, nm, f_hi);
        }
    }
}

// ---- x sweeps out of place: a warp per window of a row ------------------------
// An x line is contiguous in memory, so here the lanes run along the line: a
// warp owns a window of XW = 32 * XC positions of one row (XC consecutive
// cells per lane, one aligned vector load of F and of the face velocity),
// evaluates every stage once per position -- fluxes, Ftd, Zalesak ratios, face
// limiters, the new F -- and takes the neighbours of its first and last cell
// from the adjacent lanes by shuffle.  A stage's value is exact wherever its
// three-cell reach stays inside the window, so a window writes its positions
// XC .. XW - XC - 1 and consecutive windows of a row overlap by 2 XC.  Same
// per-cell expressions as k_fct; Fin and Fout must be different buffers.
constexpr int XC = 4, XW = 32 * XC, XOUT = XW - 2 * XC;

template <bool FINAL>
__global__ void __launch_bounds__(256) k_fct_x(Geom g, const float* __restrict__ Fin, float* __restrict__ F,
                                               const float* __restrict__ vel, int chunks) {
    constexpr unsigned FULL = 0xffffffffu;
    const Sweep<0> S(g);
    const int n = g.nx;
    const int lane = threadIdx.x & 31;
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int chunk = (int)(wid % chunks);
    const long long row = wid / chunks;
    const int j = 1 + (int)(row % g.ny), k = 1 + (int)(row / g.ny);
    if (k > g.nz) return;  // the whole warp
    const int pa = chunk * XOUT - XC;  // first position of the window
    const int x0 = pa + lane * XC;     // this lane's first position
    const int rb = gidx(g, 0, j, k);
    const float dt = S.dt;
    float Fv[XC], Vv[XC];
    if (x0 >= 0 && x0 + XC - 1 <= n + 1) {
        const float4 f4 = *reinterpret_cast<const float4*>(Fin + rb + x0);
        const float4 v4 = __ldg(reinterpret_cast<const float4*>(vel + rb + x0));
        Fv[0] = f4.x; Fv[1] = f4.y; Fv[2] = f4.z; Fv[3] = f4.w;
        Vv[0] = v4.x; Vv[1] = v4.y; Vv[2] = v4.z; Vv[3] = v4.w;
    } else {
#pragma unroll
        for (int e = 0; e < XC; ++e) {
            const int x = x0 + e;
            const bool in = x >= 0 && x <= n + 1;
            Fv[e] = in ? Fin[rb + x] : 0.0f;
            Vv[e] = in ? __ldg(vel + rb + x) : 0.0f;
        }
    }
    const int lo_out = pa + XC, hi_out = pa + XW - XC - 1;
    float out[XC];
    bool wr[XC];
#pragma unroll
    for (int e = 0; e < XC; ++e) {
        const int x = x0 + e;
        wr[e] = x >= 1 && x <= n && x >= lo_out && x <= hi_out;
        out[e] = 0.0f;
    }
    // A window where F is 0 everywhere (face velocities below vq, which keeps
    // every dv above 0.01 vol) gives 0 at each of its cells, as k_fct_march's
    // quiet positions do: most windows of a dam break are gas.
    const float vq = 0.49f * S.vol / S.dvfac;
    bool zq = true;
#pragma unroll
    for (int e = 0; e < XC; ++e) {
        const int x = x0 + e;
        zq = zq && (x < 0 || x > n + 1 || (Fv[e] == 0.0f && fabsf(Vv[e]) < vq));
    }
    if (!__all_sync(FULL, zq)) {
    // face fluxes through faces x0 .. x0+XC-1 (face x lies between cells x-1 and x)
    const float Fm = __shfl_up_sync(FULL, Fv[XC - 1], 1);
    float lo[XC], af[XC];
#pragma unroll
    for (int e = 0; e < XC; ++e) {
        const int x = x0 + e;
        lo[e] = 0.0f;
        af[e] = 0.0f;
        if (x >= 1 && x <= n + 1) fct::flux(Vv[e], e ? Fv[e - 1] : Fm, Fv[e], dt, lo[e], af[e]);
    }
    const float Vn = __shfl_down_sync(FULL, Vv[0], 1);
    const float lon = __shfl_down_sync(FULL, lo[0], 1), an = __shfl_down_sync(FULL, af[0], 1);
    // low-order update Ftd of cells x0 .. x0+XC-1 (0 outside 1..n)
    float T[XC], dv[XC], rdv[XC];
#pragma unroll
    for (int e = 0; e < XC; ++e) {
        const int x = x0 + e;
        T[e] = 0.0f;
        dv[e] = 1.0f;
        rdv[e] = 1.0f;
        if (x >= 1 && x <= n) {
            dv[e] = S.dv(Vv[e], e < XC - 1 ? Vv[e + 1] : Vn);
            rdv[e] = __frcp_rn(dv[e]);
            T[e] = ftd_from(S, Fv[e], lo[e], e < XC - 1 ? lo[e + 1] : lon, dv[e], rdv[e]);
        }
    }
    const float Tm = __shfl_up_sync(FULL, T[XC - 1], 1), Tn = __shfl_down_sync(FULL, T[0], 1);
    // Zalesak ratios (0 outside 1..n)
    float rp[XC], rm[XC];
#pragma unroll
    for (int e = 0; e < XC; ++e) {
        const int x = x0 + e;
        rp[e] = 0.0f;
        rm[e] = 0.0f;
        if (x >= 1 && x <= n)
            limiter(S, e ? T[e - 1] : Tm, T[e], e < XC - 1 ? T[e + 1] : Tn, af[e], e < XC - 1 ? af[e + 1] : an,
                    rp[e], rm[e]);
    }
    const float rpm = __shfl_up_sync(FULL, rp[XC - 1], 1), rmm = __shfl_up_sync(FULL, rm[XC - 1], 1);
    // face limiters of faces 2 .. n+1 (c[1] is never written: 0)
    float cf[XC];
#pragma unroll
    for (int e = 0; e < XC; ++e) {
        const int x = x0 + e;
        cf[e] = (x >= 2 && x <= n + 1) ? face_limit(af[e], e ? rp[e - 1] : rpm, e ? rm[e - 1] : rmm, rp[e], rm[e])
                                       : 0.0f;
    }
    const float cfn = __shfl_down_sync(FULL, cf[0], 1);
    // the new F of the window's own cells
#pragma unroll
    for (int e = 0; e < XC; ++e) {
        if (wr[e]) {
            out[e] = clamp01f(fct::stage4(S, T[e], af[e], cf[e], e < XC - 1 ? af[e + 1] : an,
                                          e < XC - 1 ? cf[e + 1] : cfn, dv[e], rdv[e]));
            if (FINAL) out[e] = clamp01f(out[e]);  // post_process_f_kernel, voftrial1.cu:502-507
        }
    }
    }  // not a quiet window
    if (!FINAL) {
        if (wr[0] && wr[1] && wr[2] && wr[3]) {
            *reinterpret_cast<float4*>(F + rb + x0) = make_float4(out[0], out[1], out[2], out[3]);
        } else {
#pragma unroll
            for (int e = 0; e < XC; ++e)
                if (wr[e]) F[rb + x0 + e] = out[e];
        }
    } else if (j > 1 && j < g.ny && k > 1 && k < g.nz) {
        // a row away from the y and z walls: only the x ghosts of the row
#pragma unroll
        for (int e = 0; e < XC; ++e) {
            if (!wr[e]) continue;
            const int x = x0 + e;
            F[rb + x] = out[e];
            if (x == 1) F[rb] = out[e];
            if (x == n) F[rb + n + 1] = out[e];
        }
    } else {
        // apply_bc_F (voftrial1.cu:1122-1135): every ghost takes the value at
        // its clamped interior index
#pragma unroll
        for (int e = 0; e < XC; ++e)
            if (wr[e]) store_mirrored(F, g.px, g.plane, g.nx, g.ny, g.nz, x0 + e, j, k, out[e]);
    }
}

static int march_resident = 4 * 148;  // blocks of k_fct_march resident at once, set by fct_configure

// Segments per line: the count (of 1 .. 16, segments of at least 16 cells)
// whose launch fills its last wave of resident blocks best, the fewest
// segments among equals (each segment start repeats a few cells of work).
static int march_segment(const Geom& g, int axis) {
    const int n = axis == 1 ? g.ny : g.nz;
    const int nb = axis == 1 ? g.nz : g.ny;
    const long long bx = ((long long)g.nx * nb + MARCH_THREADS - 1) / MARCH_THREADS;
    int best = n;
    double best_fill = -1.0;
    for (int nseg = 1; nseg <= 16; ++nseg) {
        const int seg = (n + nseg - 1) / nseg;
        if (nseg > 1 && seg < 16) break;
        const long long blocks = bx * ((n + seg - 1) / seg);
        const long long waves = (blocks + march_resident - 1) / march_resident;
        const double fill = (double)blocks / (double)(waves * march_resident);
        if (fill > best_fill + 0.02) {
            best_fill = fill;
            best = seg;
        }
    }
    return best;
}

size_t fct_smem_bytes(int axis, int n) {
    const int npos = n + 2;
    if (axis == 0) return sizeof(float) * 2u * (size_t)LANES * (size_t)odd_pitch(npos);
    return sizeof(float) * 2u * (size_t)npos * LANES;
}

template <int AXIS, bool FINAL>
static cudaError_t launch_axis(const Geom& g, const float* Fsrc, float* F, const float* vel, cudaStream_t s) {
    if (AXIS == 0 && Fsrc != F) {  // out of place along x: warps along the rows
        const int chunks = (g.nx + 1 + XOUT - 1) / XOUT;
        const long long warps = (long long)chunks * g.ny * g.nz;
        k_fct_x<FINAL><<<(unsigned)((warps + 7) / 8), 256, 0, s>>>(g, Fsrc, F, vel, chunks);
        return cudaGetLastError();
    }
    // out of place along y or z, with lines enough to fill the device (one
    // thread per line segment): the march from memory; else the tiles below
    if (AXIS != 0 && Fsrc != F && (long long)g.nx * (AXIS == 1 ? g.nz : g.ny) >= 16384) {
        constexpr int A = AXIS == 0 ? 1 : AXIS;
        const int n = A == 1 ? g.ny : g.nz, nb = A == 1 ? g.nz : g.ny;
        const int seg = march_segment(g, A);
        const dim3 grid((unsigned)(((long long)g.nx * nb + MARCH_THREADS - 1) / MARCH_THREADS),
                        (unsigned)((n + seg - 1) / seg));
        k_fct_march<A, FINAL><<<grid, MARCH_THREADS, 0, s>>>(g, Fsrc, F, vel, seg);
        return cudaGetLastError();
    }
    const int n = AXIS == 0 ? g.nx : (AXIS == 1 ? g.ny : g.nz);
    const int na = AXIS == 0 ? g.ny : g.nx;
    const int nb = AXIS == 2 ? g.ny : g.nz;
    dim3 grid((na * nb + LANES - 1) / LANES, 1, 1);
    k_fct<AXIS, FINAL><<<grid, dim3(LANES, WARPS), fct_smem_bytes(AXIS, n), s>>>(g, Fsrc, F, vel);
    return cudaGetLastError();
}

cudaError_t fct_launch_to(const Geom& g, int axis, bool final_sweep, const float* Fin, float* Fout, const float* vel,
                          cudaStream_t s) {
    if (axis == 0)
        return final_sweep ? launch_axis<0, true>(g, Fin, Fout, vel, s) : launch_axis<0, false>(g, Fin, Fout, vel, s);
    if (axis == 1)
        return final_sweep ? launch_axis<1, true>(g, Fin, Fout, vel, s) : launch_axis<1, false>(g, Fin, Fout, vel, s);
    return final_sweep ? launch_axis<2, true>(g, Fin, Fout, vel, s) : launch_axis<2, false>(g, Fin, Fout, vel, s);
}

cudaError_t fct_launch(const Geom& g, int axis, bool final_sweep, float* F, const float* vel, cudaStream_t s) {
    return fct_launch_to(g, axis, final_sweep, F, F, vel, s);
}

cudaError_t fct_configure() {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
#define VOF_SET(A, FIN)                                                                      \
    if ((e = cudaFuncSetAttribute(k_fct<A, FIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  optin)) != cudaSuccess)                                    \
        return e;
    VOF_SET(0, false) VOF_SET(0, true) VOF_SET(1, false) VOF_SET(1, true) VOF_SET(2, false) VOF_SET(2, true)
#undef VOF_SET
    int sms = 0, occ = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fct_march<2, false>, MARCH_THREADS, 0)) !=
            cudaSuccess)
        return e;
    march_resident = (sms > 0 ? sms : 148) * (occ > 0 ? occ : 1);
    return cudaSuccess;
}

size_t fct_smem_limit() { return 227u * 1024u; }

}  // namespace vof
