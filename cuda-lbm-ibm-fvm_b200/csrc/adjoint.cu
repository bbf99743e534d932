// adjoint.cu -- reverse mode of the plain step on the device (extension; the
// reference has no adjoint).  Compiled with -fmad=false: the FP32 forward
// values recomputed here (FCT stages, advecting velocities, clamps) are the
// forward's own bits, so every switch of the reverse pass is the one the
// forward took.  Adjoint fields are FP64.
//
// Derivative conventions (the same as the host adjoint in the oracle): a
// branch differentiates the side it took; fmaxf / fminf differentiate the
// argument they returned, the first on a tie; clamp01f has derivative 1 on
// [0, 1] and 0 outside.
//
// Per reversed step (voftrial1.cu:1364-1401 backwards):
//   recompute: predictor + rhs, the Jacobi sweeps, the velocity correction,
//     F before sweeps 2 and 3 (the forward's own kernels);
//   F boundary copies (voftrial1.cu:1053-1135) reversed;
//   each FCT sweep reversed (voftrial1.cu:509-905): its stages recomputed
//     cell by cell, then five gather kernels (stage 4; the limiter and
//     stage 2's ratios; stage 2's extrema and stage 1; the face fluxes and
//     velocities; F) -- no atomics;
//   velocity boundary copies (voftrial1.cu:959-1051) reversed;
//   velocity correction (voftrial1.cu:441-493) reversed (atomics into the
//     pressure and density adjoints);
//   Jacobi sweeps transposed (voftrial1.cu:401-439): mu = lambda / ap,
//     lrhs += mu, lambda' = -N mu, one gather kernel per sweep;
//   rhs (voftrial1.cu:418-422) reversed, gather;
//   advection (voftrial1.cu:230-399) reversed (atomics), dL/dg per block;
//   rho and nu (voftrial1.cu:95-104) reversed.
#include <cuda_runtime.h>
#include <math.h>

#include <stdlib.h>
#include <string.h>

#include <initializer_list>
#include <new>
#include <utility>

#include "adjoint.h"
#include "fct_line.cuh"
#include "fct_sweep.h"
#include "jacobi_tb.h"

namespace vof {

namespace {

struct Range {
    int i0, i1, j0, j1, k0, k1;  // inclusive
};

constexpr int AB_X = 32, AB_Y = 4, AB_Z = 2;

inline dim3 grid_of(const Range& r) {
    return dim3((r.i1 - r.i0 + AB_X) / AB_X, (r.j1 - r.j0 + AB_Y) / AB_Y, (r.k1 - r.k0 + AB_Z) / AB_Z);
}
const dim3 kBlk(AB_X, AB_Y, AB_Z);

#define RANGE_CELL(R)                                              \
    const int i = (R).i0 + blockIdx.x * blockDim.x + threadIdx.x; \
    const int j = (R).j0 + blockIdx.y * blockDim.y + threadIdx.y; \
    const int k = (R).k0 + blockIdx.z * blockDim.z + threadIdx.z; \
    if (i > (R).i1 || j > (R).j1 || k > (R).k1) return

inline Range interior(const Geom& g) { return {1, g.nx, 1, g.ny, 1, g.nz}; }

// The sweep axis DIR: unit offset, position along it, line length.
template <int DIR>
__device__ __forceinline__ int sstride(const Geom& g) {
    return DIR == 0 ? 1 : (DIR == 1 ? g.px : g.plane);
}
template <int DIR>
__device__ __forceinline__ int spos(int i, int j, int k) {
    return DIR == 0 ? i : (DIR == 1 ? j : k);
}
template <int DIR>
__device__ __forceinline__ int slen(const Geom& g) {
    return DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
}
template <int DIR>
__device__ __forceinline__ float dvfac_of(const Geom& g) {
    return DIR == 0 ? g.dt * g.dy * g.dz : (DIR == 1 ? g.dt * g.dx * g.dz : g.dt * g.dx * g.dy);
}
__device__ __forceinline__ float lowflux(const Geom& g, const float* vel, const float* F, int f, int cm, int cp) {
    const float uf = vel[f];
    return (uf >= 0.0f) ? uf * g.dt * F[cm] : uf * g.dt * F[cp];
}
__device__ __forceinline__ float highflux(const Geom& g, const float* vel, const float* F, int f, int cm, int cp) {
    const float uf = vel[f];
    return (uf <= 0.0f) ? uf * g.dt * F[cm] : uf * g.dt * F[cp];
}

// ---- FCT stages, cell by cell (the expressions of fct_x/y/z_sweep_stage1..3) -----
template <int DIR>
__global__ void __launch_bounds__(256) k_fs1(Geom g, Range R, const float* __restrict__ F,
                                             const float* __restrict__ vel, float* __restrict__ Ftd) {
    RANGE_CELL(R);
    const int s = sstride<DIR>(g), c = gidx(g, i, j, k);
    const float vol = g.dx * g.dy * g.dz;
    const float dv = vol - dvfac_of<DIR>(g) * (vel[c + s] - vel[c]);
    const float f_in = lowflux(g, vel, F, c, c - s, c);
    const float f_out = lowflux(g, vel, F, c + s, c, c + s);
    float term;
    if (DIR == 0) term = (f_in - f_out) * g.dy * g.dz / vol;
    else if (DIR == 1) term = (f_in - f_out) * g.dy / (g.dx * g.dy);
    else term = (f_in - f_out) * g.dy * g.dx / vol;
    float out = (F[c] + term) * vol / dv;
    if (out > 1.0f || out < 0.0f) out = clamp01f(out);
    Ftd[c] = out;
}

// A at the lower face of every cell (and the upper face of the last), rp, rm.
template <int DIR>
__global__ void __launch_bounds__(256) k_fs2(Geom g, Range R, const float* __restrict__ F,
                                             const float* __restrict__ vel, const float* __restrict__ Ftd,
                                             float* __restrict__ A, float* __restrict__ rp, float* __restrict__ rm) {
    RANGE_CELL(R);
    const int s = sstride<DIR>(g), c = gidx(g, i, j, k);
    const float a1 = highflux(g, vel, F, c + s, c, c + s) - lowflux(g, vel, F, c + s, c, c + s);
    const float a0 = highflux(g, vel, F, c, c - s, c) - lowflux(g, vel, F, c, c - s, c);
    A[c] = a0;
    if (spos<DIR>(i, j, k) == slen<DIR>(g)) A[c + s] = a1;
    const float pp = fmaxf(0.0f, a0) - fminf(0.0f, a1);
    const float pm = fmaxf(0.0f, a1) - fminf(0.0f, a0);
    const float fmx = fmaxf(Ftd[c], fmaxf(Ftd[c - s], Ftd[c + s]));
    const float fmn = fminf(Ftd[c], fminf(Ftd[c - s], Ftd[c + s]));
    const float hq = DIR == 2 ? g.dz : g.dx;
    const float qp = (fmx - Ftd[c]) * hq;
    rp[c] = (pp > 0.0f) ? fminf(1.0f, qp / pp) : 0.0f;
    const float qm = (Ftd[c] - fmn) * hq;
    rm[c] = (pm > 0.0f) ? fminf(1.0f, qm / pm) : 0.0f;
}

// The limiter at the upper face of every cell; 0 at the first face (never
// written by the reference's stage 3).
template <int DIR>
__global__ void __launch_bounds__(256) k_fs3(Geom g, Range R, const float* __restrict__ A,
                                             const float* __restrict__ rp, const float* __restrict__ rm,
                                             float* __restrict__ C) {
    RANGE_CELL(R);
    const int s = sstride<DIR>(g), c = gidx(g, i, j, k);
    C[c + s] = (A[c + s] >= 0.0f) ? fminf(rp[c + s], rm[c]) : fminf(rp[c], rm[c + s]);
    if (spos<DIR>(i, j, k) == 1) C[c] = 0.0f;
}

// Adjoint, part 0 (per interior cell): stage 4.  out = Ftd - X vol / dv,
// X = (A1 C1 - A0 C0) / K4, F = clamp01f(out): g4 = lF * (clamp derivative)
// is the adjoint of Ftd through stage 4; lX = -g4 vol / dv the adjoint of X;
// ldv (stage-4 part) = g4 X vol / dv^2.
template <int DIR>
__global__ void __launch_bounds__(256) k_as4(Geom g, Range R, const float* __restrict__ vel,
                                             const float* __restrict__ Ftd, const float* __restrict__ A,
                                             const float* __restrict__ C, const double* __restrict__ lF,
                                             double* __restrict__ lX, double* __restrict__ ldv,
                                             double* __restrict__ lown) {
    RANGE_CELL(R);
    const int s = sstride<DIR>(g), c = gidx(g, i, j, k);
    const float vol = g.dx * g.dy * g.dz;
    const float dv = vol - dvfac_of<DIR>(g) * (vel[c + s] - vel[c]);
    const float K4 = DIR == 2 ? g.dz : g.dy;
    const float a0 = A[c], a1 = A[c + s], c0 = C[c], c1 = C[c + s];
    const float out = Ftd[c] - ((a1 * c1 - a0 * c0) / K4) * vol / dv;
    const double g4 = (out >= 0.0f && out <= 1.0f) ? lF[c] : 0.0;
    const double idv = 1.0 / (double)dv, vold = (double)vol;
    const double X = ((double)a1 * c1 - (double)a0 * c0) / (double)K4;
    lX[c] = -g4 * vold * idv;
    ldv[c] = g4 * X * vold * idv * idv;
    lown[c] = g4;
}

// Adjoint, part 1 (per interior cell): the limiter (stage 3) and the limiter
// ratios (stage 2).  Stores the extremum adjoints with the cells they
// selected, lpp / lpm, and adds the direct stage-2 terms to lown (the
// adjoint of Ftd[c] from its own cell).
template <int DIR>
__global__ void __launch_bounds__(256) k_as3(Geom g, Range R, const float* __restrict__ Ftd,
                                             const float* __restrict__ A, const float* __restrict__ rp,
                                             const float* __restrict__ rm, const double* __restrict__ lX,
                                             double* __restrict__ lmx, double* __restrict__ lmn,
                                             double* __restrict__ lpp, double* __restrict__ lpm,
                                             double* __restrict__ lown, unsigned char* __restrict__ sel) {
    RANGE_CELL(R);
    const int s = sstride<DIR>(g), c = gidx(g, i, j, k);
    const int pos = spos<DIR>(i, j, k), n = slen<DIR>(g);
    const double iK4 = 1.0 / (DIR == 2 ? (double)g.dz : (double)g.dy);
    const double lXc = lX[c];
    const double lXm = pos >= 2 ? lX[c - s] : 0.0;
    const double lXp = pos <= n - 1 ? lX[c + s] : 0.0;
    const float a0 = A[c], a1 = A[c + s];
    // limiter: faces c (lower) and c + s (upper)
    const double lC_hi = (lXc - lXp) * (double)a1 * iK4;
    const double lC_lo = pos >= 2 ? (lXm - lXc) * (double)a0 * iK4 : 0.0;
    double lrp = 0.0, lrm = 0.0;
    if (pos >= 2) {
        if (a0 >= 0.0f) {
            if (rp[c] <= rm[c - s]) lrp += lC_lo;
        } else {
            if (!(rp[c - s] <= rm[c])) lrm += lC_lo;
        }
    }
    if (a1 >= 0.0f) {
        if (!(rp[c + s] <= rm[c])) lrm += lC_hi;
    } else {
        if (rp[c] <= rm[c + s]) lrp += lC_hi;
    }
    // limiter ratios
    const float pp = fmaxf(0.0f, a0) - fminf(0.0f, a1);
    const float pm = fmaxf(0.0f, a1) - fminf(0.0f, a0);
    const float fc = Ftd[c], fl = Ftd[c - s], fh = Ftd[c + s];
    const float hqf = DIR == 2 ? g.dz : g.dx;
    const double hq = (double)hqf;
    double lqp = 0.0, lqm = 0.0, dpp = 0.0, dpm = 0.0;
    if (lrp != 0.0) {
        const float qp = (fmaxf(fc, fmaxf(fl, fh)) - fc) * hqf;
        if (pp > 0.0f && qp / pp < 1.0f) {
            const double ip = 1.0 / (double)pp;
            lqp = lrp * ip;
            dpp = -lqp * (double)qp * ip;
        }
    }
    if (lrm != 0.0) {
        const float qm = (fc - fminf(fc, fminf(fl, fh))) * hqf;
        if (pm > 0.0f && qm / pm < 1.0f) {
            const double ip = 1.0 / (double)pm;
            lqm = lrm * ip;
            dpm = -lqm * (double)qm * ip;
        }
    }
    const int in_mx = (fl >= fh) ? 0 : 2;  // 0: c - s, 1: c, 2: c + s
    const int smx = (fc >= (in_mx == 0 ? fl : fh)) ? 1 : in_mx;
    const int in_mn = (fl <= fh) ? 0 : 2;
    const int smn = (fc <= (in_mn == 0 ? fl : fh)) ? 1 : in_mn;
    lmx[c] = lqp * hq;
    lmn[c] = -lqm * hq;
    sel[c] = (unsigned char)(smx | (smn << 2));
    lpp[c] = dpp;
    lpm[c] = dpm;
    lown[c] += -lqp * hq + lqm * hq;
}

// Adjoint, part 2 (per interior cell): the full adjoint of Ftd[c] (own terms
// and the neighbours' extrema that selected c), then stage 1: lterm = the
// adjoint of the stage-1 flux difference (and of F[c] through it), ldv total.
template <int DIR>
__global__ void __launch_bounds__(256) k_as2(Geom g, Range R, const float* __restrict__ F,
                                             const float* __restrict__ vel, const double* __restrict__ lmx,
                                             const double* __restrict__ lmn, const unsigned char* __restrict__ sel,
                                             const double* __restrict__ lown, double* __restrict__ ldv,
                                             double* __restrict__ lterm) {
    RANGE_CELL(R);
    const int s = sstride<DIR>(g), c = gidx(g, i, j, k);
    const int pos = spos<DIR>(i, j, k), n = slen<DIR>(g);
    double lFtd = lown[c];
    for (int d = -1; d <= 1; ++d) {
        if (pos + d < 1 || pos + d > n) continue;
        const int e = c + d * s;
        const int sb = sel[e];
        const int want = 1 - d;  // e's slot (0, 1, 2 = e - s, e, e + s) that is c
        if ((sb & 3) == want) lFtd += lmx[e];
        if ((sb >> 2) == want) lFtd += lmn[e];
    }
    const float vol = g.dx * g.dy * g.dz;
    const float dv = vol - dvfac_of<DIR>(g) * (vel[c + s] - vel[c]);
    const float f_in = lowflux(g, vel, F, c, c - s, c);
    const float f_out = lowflux(g, vel, F, c + s, c, c + s);
    float term;
    if (DIR == 0) term = (f_in - f_out) * g.dy * g.dz / vol;
    else if (DIR == 1) term = (f_in - f_out) * g.dy / (g.dx * g.dy);
    else term = (f_in - f_out) * g.dy * g.dx / vol;
    const float out = (F[c] + term) * vol / dv;
    const double h = (out > 1.0f || out < 0.0f) ? 0.0 : lFtd;
    const double dvd = (double)dv, vold = (double)vol;
    lterm[c] = h * vold / dvd;
    ldv[c] -= h * ((double)F[c] + (double)term) * vold / (dvd * dvd);
}

// Adjoint, part 3 (per face: positions 1 .. n+1 along the axis, the face
// being the lower face of cell f): the low-order flux LF_f and the
// antidiffusive flux A_f, and the face velocity.
template <int DIR>
__global__ void __launch_bounds__(256) k_as1(Geom g, Range R, const float* __restrict__ F,
                                             const float* __restrict__ vel, const float* __restrict__ A,
                                             const float* __restrict__ C, const double* __restrict__ lX,
                                             const double* __restrict__ lpp, const double* __restrict__ lpm,
                                             const double* __restrict__ ldv, const double* __restrict__ lterm,
                                             double* __restrict__ lLF, double* __restrict__ lA,
                                             double* __restrict__ lvel) {
    RANGE_CELL(R);
    const int s = sstride<DIR>(g), f = gidx(g, i, j, k);
    const int pos = spos<DIR>(i, j, k), n = slen<DIR>(g);
    const bool lo = pos >= 2, hi = pos <= n;  // cells f - s and f are interior
    const double vol = (double)(g.dx * g.dy * g.dz);
    const double K1 = DIR == 0 ? (double)g.dy * g.dz / vol
                               : (DIR == 1 ? (double)g.dy / ((double)g.dx * g.dy) : (double)g.dy * g.dx / vol);
    const double K4 = DIR == 2 ? (double)g.dz : (double)g.dy;
    const double dt = (double)g.dt;
    const float a = A[f];
    const double l_LF = K1 * ((hi ? lterm[f] : 0.0) - (lo ? lterm[f - s] : 0.0));
    double l_A = ((lo ? lX[f - s] : 0.0) - (hi ? lX[f] : 0.0)) * (double)C[f] / K4;
    if (hi) l_A += (a > 0.0f ? lpp[f] : 0.0) - (a < 0.0f ? lpm[f] : 0.0);
    if (lo) l_A += -(a < 0.0f ? lpp[f - s] : 0.0) + (a > 0.0f ? lpm[f - s] : 0.0);
    const float uf = vel[f];
    const int hs = (uf <= 0.0f) ? f - s : f;
    const int ls = (uf >= 0.0f) ? f - s : f;
    lvel[f] += l_LF * dt * (double)F[ls] + l_A * dt * ((double)F[hs] - (double)F[ls]) +
               (double)dvfac_of<DIR>(g) * ((hi ? ldv[f] : 0.0) - (lo ? ldv[f - s] : 0.0));
    lLF[f] = l_LF;
    lA[f] = l_A;
}

// Adjoint, part 4 (per cell: positions 0 .. n+1 along the axis): the adjoint
// of the sweep's input F (the ghosts keep theirs: the sweep does not write them).
template <int DIR>
__global__ void __launch_bounds__(256) k_as0(Geom g, Range R, const float* __restrict__ vel,
                                             const double* __restrict__ lterm, const double* __restrict__ lLF,
                                             const double* __restrict__ lA, double* __restrict__ lF) {
    RANGE_CELL(R);
    const int s = sstride<DIR>(g), c = gidx(g, i, j, k);
    const int pos = spos<DIR>(i, j, k), n = slen<DIR>(g);
    const double dt = (double)g.dt;
    double acc = (pos >= 1 && pos <= n) ? lterm[c] : lF[c];
    if (pos >= 1) {  // face c: cell c is its upper cell
        const float uf = vel[c];
        const double w = (double)uf * dt;
        if (uf < 0.0f) acc += lLF[c] * w;                          // lowflux took F[c]
        acc += lA[c] * w * ((uf > 0.0f ? 1.0 : 0.0) - (uf < 0.0f ? 1.0 : 0.0));
    }
    if (pos <= n) {  // face c + s: cell c is its lower cell
        const float uf = vel[c + s];
        const double w = (double)uf * dt;
        if (uf >= 0.0f) acc += lLF[c + s] * w;
        acc += lA[c + s] * w * ((uf <= 0.0f ? 1.0 : 0.0) - (uf >= 0.0f ? 1.0 : 0.0));
    }
    lF[c] = acc;
}

// ---- the whole sweep adjoint in one kernel, LPB lines per block in shared memory ----
// The same quantities as k_fs1..3 and k_as4..0, staged per line in shared
// memory (positions 0 .. n+1 of LPB lines), one phase per __syncthreads: load,
// the three forward stages (the forward's expressions), stage 4's adjoint,
// the limiter and stage 2's ratios, stage 2's extrema and stage 1, the faces,
// F.  Global traffic: F, vel and lF read once, lF and lvel written once.
// Thread mapping: DIR 0 (x lines): a line's positions run over consecutive
// threads (coalesced along x); DIR 1/2: LPB x-adjacent lines per block, the
// line index fastest (LPB consecutive floats per position).
constexpr int FA_THREADS = 256;
__host__ __device__ __forceinline__ size_t fa_smem_bytes(int lpb, int n) {
    const size_t m = (size_t)lpb * (n + 2);
    return m * (7 * sizeof(double) + 7 * sizeof(float) + 1);
}
template <int DIR, int LPB>
__global__ void __launch_bounds__(FA_THREADS) k_fct_adjoint(Geom g, const float* __restrict__ Fg,
                                                            const float* __restrict__ velg, double* __restrict__ lFg,
                                                            double* __restrict__ lvelg) {
    extern __shared__ __align__(16) unsigned char fa_smem[];
    const int n = slen<DIR>(g), N2 = n + 2, M = LPB * N2;
    double* sLX = reinterpret_cast<double*>(fa_smem);
    double* sLdv = sLX + M;
    double* sLmx = sLdv + M;   // later: the adjoint of the low-order flux at each face
    double* sLmn = sLmx + M;   // later: the adjoint of A at each face
    double* sLpp = sLmn + M;
    double* sLpm = sLpp + M;
    double* sLown = sLpm + M;  // later (P6, in place): lterm
    double* sLterm = sLown;
    float* sF = reinterpret_cast<float*>(sLown + M);
    float* sV = sF + M;
    float* sFtd = sV + M;
    float* sA = sFtd + M;
    float* sRp = sA + M;
    float* sRm = sRp + M;
    float* sC = sRm + M;
    unsigned char* sSel = reinterpret_cast<unsigned char*>(sC + M);

    constexpr int TPL = FA_THREADS / LPB;  // threads per line
    const int tid = threadIdx.x;
    const int l = DIR == 0 ? tid / TPL : tid % LPB;
    const int p0 = DIR == 0 ? tid % TPL : tid / LPB;
    // this thread's line: global base (position 0) and stride along the axis
    int base, gs;
    bool act;
    if (DIR == 0) {
        const int j = 1 + blockIdx.x * LPB + l, k = 1 + blockIdx.y;
        act = j <= g.ny;
        base = gidx(g, 0, act ? j : 1, k);
        gs = 1;
    } else if (DIR == 1) {
        const int i = 1 + blockIdx.x * LPB + l, k = 1 + blockIdx.y;
        act = i <= g.nx;
        base = gidx(g, act ? i : 1, 0, k);
        gs = g.px;
    } else {
        const int i = 1 + blockIdx.x * LPB + l, j = 1 + blockIdx.y;
        act = i <= g.nx;
        base = gidx(g, act ? i : 1, j, 0);
        gs = g.plane;
    }
    auto si = [&](int q) { return DIR == 0 ? l * N2 + q : q * LPB + l; };
    const float vol = g.dx * g.dy * g.dz;
    const float dvfac = dvfac_of<DIR>(g);
    const float K4 = DIR == 2 ? g.dz : g.dy;
    const float hqf = DIR == 2 ? g.dz : g.dx;
    const double vold = (double)vol, dt = (double)g.dt, iK4 = 1.0 / (double)K4, hq = (double)hqf;
    const double K1 = DIR == 0 ? (double)g.dy * g.dz / vold
                               : (DIR == 1 ? (double)g.dy / ((double)g.dx * g.dy) : (double)g.dy * g.dx / vold);

    // P0: load
    if (act)
        for (int q = p0; q < N2; q += TPL) {
            const int c = base + q * gs;
            sF[si(q)] = Fg[c];
            sV[si(q)] = q >= 1 ? velg[c] : 0.0f;
        }
    __syncthreads();
    // P1: stage 1 (Ftd; 0 at the ghosts)
    if (act)
        for (int q = p0; q < N2; q += TPL) {
            if (q == 0 || q == n + 1) {
                sFtd[si(q)] = 0.0f;
                continue;
            }
            const float vl = sV[si(q)], vh = sV[si(q + 1)];
            const float dv = vol - dvfac * (vh - vl);
            const float f_in = (vl >= 0.0f) ? vl * g.dt * sF[si(q - 1)] : vl * g.dt * sF[si(q)];
            const float f_out = (vh >= 0.0f) ? vh * g.dt * sF[si(q)] : vh * g.dt * sF[si(q + 1)];
            float term;
            if (DIR == 0) term = (f_in - f_out) * g.dy * g.dz / vol;
            else if (DIR == 1) term = (f_in - f_out) * g.dy / (g.dx * g.dy);
            else term = (f_in - f_out) * g.dy * g.dx / vol;
            float out = (sF[si(q)] + term) * vol / dv;
            if (out > 1.0f || out < 0.0f) out = clamp01f(out);
            sFtd[si(q)] = out;
        }
    __syncthreads();
    // P2: stage 2 (A at the lower face of every cell and the last upper face; rp, rm)
    if (act)
        for (int q = p0; q < N2; q += TPL) {
            if (q == 0 || q == n + 1) {
                sRp[si(q)] = 0.0f;
                sRm[si(q)] = 0.0f;
                continue;
            }
            const float vl = sV[si(q)], vh = sV[si(q + 1)];
            const float Fm = sF[si(q - 1)], Fc = sF[si(q)], Fp = sF[si(q + 1)];
            const float a1 = ((vh <= 0.0f) ? vh * g.dt * Fc : vh * g.dt * Fp) -
                             ((vh >= 0.0f) ? vh * g.dt * Fc : vh * g.dt * Fp);
            const float a0 = ((vl <= 0.0f) ? vl * g.dt * Fm : vl * g.dt * Fc) -
                             ((vl >= 0.0f) ? vl * g.dt * Fm : vl * g.dt * Fc);
            sA[si(q)] = a0;
            if (q == n) sA[si(q + 1)] = a1;
            const float pp = fmaxf(0.0f, a0) - fminf(0.0f, a1);
            const float pm = fmaxf(0.0f, a1) - fminf(0.0f, a0);
            const float fc = sFtd[si(q)], fl = sFtd[si(q - 1)], fh = sFtd[si(q + 1)];
            const float fmx = fmaxf(fc, fmaxf(fl, fh));
            const float fmn = fminf(fc, fminf(fl, fh));
            const float qp = (fmx - fc) * hqf;
            sRp[si(q)] = (pp > 0.0f) ? fminf(1.0f, qp / pp) : 0.0f;
            const float qm = (fc - fmn) * hqf;
            sRm[si(q)] = (pm > 0.0f) ? fminf(1.0f, qm / pm) : 0.0f;
        }
    __syncthreads();
    // P3: stage 3 (C at the upper face of every cell; 0 at the first face)
    if (act)
        for (int q = p0; q < N2; q += TPL) {
            if (q == 0 || q == n + 1) continue;
            const int f = q + 1;
            sC[si(f)] = (sA[si(f)] >= 0.0f) ? fminf(sRp[si(f)], sRm[si(q)]) : fminf(sRp[si(q)], sRm[si(f)]);
            if (q == 1) sC[si(1)] = 0.0f;
        }
    __syncthreads();
    // P4: stage 4 reversed: g4, lX, the stage-4 part of ldv
    if (act)
        for (int q = p0; q < N2; q += TPL) {
            if (q == 0 || q == n + 1) {
                sLX[si(q)] = 0.0;
                continue;
            }
            const float dv = vol - dvfac * (sV[si(q + 1)] - sV[si(q)]);
            const float a0 = sA[si(q)], a1 = sA[si(q + 1)], c0 = sC[si(q)], c1 = sC[si(q + 1)];
            const float out = sFtd[si(q)] - ((a1 * c1 - a0 * c0) / K4) * vol / dv;
            const double g4 = (out >= 0.0f && out <= 1.0f) ? lFg[base + q * gs] : 0.0;
            const double idv = 1.0 / (double)dv;
            const double X = ((double)a1 * c1 - (double)a0 * c0) * iK4;
            sLX[si(q)] = -g4 * vold * idv;
            sLdv[si(q)] = g4 * X * vold * idv * idv;
            sLown[si(q)] = g4;
        }
    __syncthreads();
    // P5: limiter (stage 3) and limiter ratios (stage 2) reversed
    if (act)
        for (int q = p0; q < N2; q += TPL) {
            if (q == 0 || q == n + 1) continue;
            const double lXc = sLX[si(q)], lXm = sLX[si(q - 1)], lXp = sLX[si(q + 1)];
            const float a0 = sA[si(q)], a1 = sA[si(q + 1)];
            const double lC_hi = (lXc - lXp) * (double)a1 * iK4;
            const double lC_lo = q >= 2 ? (lXm - lXc) * (double)a0 * iK4 : 0.0;
            double lrp = 0.0, lrm = 0.0;
            if (q >= 2) {
                if (a0 >= 0.0f) {
                    if (sRp[si(q)] <= sRm[si(q - 1)]) lrp += lC_lo;
                } else {
                    if (!(sRp[si(q - 1)] <= sRm[si(q)])) lrm += lC_lo;
                }
            }
            if (a1 >= 0.0f) {
                if (!(sRp[si(q + 1)] <= sRm[si(q)])) lrm += lC_hi;
            } else {
                if (sRp[si(q)] <= sRm[si(q + 1)]) lrp += lC_hi;
            }
            const float pp = fmaxf(0.0f, a0) - fminf(0.0f, a1);
            const float pm = fmaxf(0.0f, a1) - fminf(0.0f, a0);
            const float fc = sFtd[si(q)], fl = sFtd[si(q - 1)], fh = sFtd[si(q + 1)];
            double lqp = 0.0, lqm = 0.0, dpp = 0.0, dpm = 0.0;
            if (lrp != 0.0) {
                const float qp = (fmaxf(fc, fmaxf(fl, fh)) - fc) * hqf;
                if (pp > 0.0f && qp / pp < 1.0f) {
                    const double ip = 1.0 / (double)pp;
                    lqp = lrp * ip;
                    dpp = -lqp * (double)qp * ip;
                }
            }
            if (lrm != 0.0) {
                const float qm = (fc - fminf(fc, fminf(fl, fh))) * hqf;
                if (pm > 0.0f && qm / pm < 1.0f) {
                    const double ip = 1.0 / (double)pm;
                    lqm = lrm * ip;
                    dpm = -lqm * (double)qm * ip;
                }
            }
            const int in_mx = (fl >= fh) ? 0 : 2;
            const int smx = (fc >= (in_mx == 0 ? fl : fh)) ? 1 : in_mx;
            const int in_mn = (fl <= fh) ? 0 : 2;
            const int smn = (fc <= (in_mn == 0 ? fl : fh)) ? 1 : in_mn;
            sLmx[si(q)] = lqp * hq;
            sLmn[si(q)] = -lqm * hq;
            sSel[si(q)] = (unsigned char)(smx | (smn << 2));
            sLpp[si(q)] = dpp;
            sLpm[si(q)] = dpm;
            sLown[si(q)] += -lqp * hq + lqm * hq;
        }
    __syncthreads();
    // P6: the adjoint of Ftd (own terms and the neighbours' extrema), stage 1 reversed
    if (act)
        for (int q = p0; q < N2; q += TPL) {
            if (q == 0 || q == n + 1) {
                sLterm[si(q)] = 0.0;  // (sLown of a ghost is never read)
                continue;
            }
            double lFtd = sLown[si(q)];
            for (int d = -1; d <= 1; ++d) {
                const int e = q + d;
                if (e < 1 || e > n) continue;
                const int sb = sSel[si(e)];
                const int want = 1 - d;
                if ((sb & 3) == want) lFtd += sLmx[si(e)];
                if ((sb >> 2) == want) lFtd += sLmn[si(e)];
            }
            const float vl = sV[si(q)], vh = sV[si(q + 1)];
            const float dv = vol - dvfac * (vh - vl);
            const float f_in = (vl >= 0.0f) ? vl * g.dt * sF[si(q - 1)] : vl * g.dt * sF[si(q)];
            const float f_out = (vh >= 0.0f) ? vh * g.dt * sF[si(q)] : vh * g.dt * sF[si(q + 1)];
            float term;
            if (DIR == 0) term = (f_in - f_out) * g.dy * g.dz / vol;
            else if (DIR == 1) term = (f_in - f_out) * g.dy / (g.dx * g.dy);
            else term = (f_in - f_out) * g.dy * g.dx / vol;
            const float out = (sF[si(q)] + term) * vol / dv;
            const double h = (out > 1.0f || out < 0.0f) ? 0.0 : lFtd;
            const double dvd = (double)dv;
            sLterm[si(q)] = h * vold / dvd;
            sLdv[si(q)] -= h * ((double)sF[si(q)] + (double)term) * vold / (dvd * dvd);
        }
    __syncthreads();
    // P7: faces 1 .. n+1 (the lower face of position q): LF and A reversed, the face velocity
    if (act)
        for (int q = p0; q < N2; q += TPL) {
            if (q == 0) continue;
            const bool lo = q >= 2, hi = q <= n;
            const float a = sA[si(q)];
            const double l_LF = K1 * ((hi ? sLterm[si(q)] : 0.0) - (lo ? sLterm[si(q - 1)] : 0.0));
            double l_A = ((lo ? sLX[si(q - 1)] : 0.0) - (hi ? sLX[si(q)] : 0.0)) * (double)sC[si(q)] * iK4;
            if (hi) l_A += (a > 0.0f ? sLpp[si(q)] : 0.0) - (a < 0.0f ? sLpm[si(q)] : 0.0);
            if (lo) l_A += -(a < 0.0f ? sLpp[si(q - 1)] : 0.0) + (a > 0.0f ? sLpm[si(q - 1)] : 0.0);
            const float uf = sV[si(q)];
            const float Fh = (uf <= 0.0f) ? sF[si(q - 1)] : sF[si(q)];
            const float Fl = (uf >= 0.0f) ? sF[si(q - 1)] : sF[si(q)];
            lvelg[base + q * gs] += l_LF * dt * (double)Fl + l_A * dt * ((double)Fh - (double)Fl) +
                                    (double)dvfac * ((hi ? sLdv[si(q)] : 0.0) - (lo ? sLdv[si(q - 1)] : 0.0));
            sLmx[si(q)] = l_LF;  // the extremum adjoints were last read in P6
            sLmn[si(q)] = l_A;
        }
    __syncthreads();
    // P8: the adjoint of the sweep's input F (ghosts keep theirs)
    if (act)
        for (int q = p0; q < N2; q += TPL) {
            double acc = (q >= 1 && q <= n) ? sLterm[si(q)] : lFg[base + q * gs];
            if (q >= 1) {  // face q: this cell is its upper cell
                const float uf = sV[si(q)];
                const double w = (double)uf * dt;
                if (uf < 0.0f) acc += sLmx[si(q)] * w;
                acc += sLmn[si(q)] * w * ((uf > 0.0f ? 1.0 : 0.0) - (uf < 0.0f ? 1.0 : 0.0));
            }
            if (q <= n) {  // face q + 1: this cell is its lower cell
                const float uf = sV[si(q + 1)];
                const double w = (double)uf * dt;
                if (uf >= 0.0f) acc += sLmx[si(q + 1)] * w;
                acc += sLmn[si(q + 1)] * w * ((uf <= 0.0f ? 1.0 : 0.0) - (uf >= 0.0f ? 1.0 : 0.0));
            }
            lFg[base + q * gs] = acc;
        }
}

// ---- the sweep adjoint as one march along each line, one lane per line ------------
// A block owns FM_LANES lines (one per lane, numbered over both cross axes)
// and splits each line's positions 0 .. n+1 into WARPS segments, one per warp.  A warp walks its segment once,
// starting FM_WARM positions early; iteration c evaluates, in registers, the
// forward and reverse stages at staggered positions, each from values that
// earlier stages or iterations produced:
//   s1  face c+6 fluxes, cell c+5 Ftd (stage 1)    s6  cell c+2: limiter ratios reversed
//   s2  cell c+4 ratios rp, rm (stage 2)           s7  cell c+1: adjoint of Ftd complete, stage 1 reversed
//   s3  face c+4 limiter C (stage 3)               s8  face c+1: adjoint of its fluxes and its velocity
//   s4  cell c+3: stage 4 reversed (reads lF)      s9  cell c: adjoint of the sweep's input F
//   s5  face c+3: the limiter's adjoint, routed to the cell whose ratio it took
// Adjoint contributions are added where they arise into short windows of
// accumulators (per cell: lrp, lrm, the adjoint of Ftd, of dv, of the input
// F; per face: of A).  The forward values are the forward kernel's own
// expressions (fct_line.cuh), so every switch is the forward's.  The warm-up
// positions recompute what the previous segment also computes and write
// nothing; FM_WARM = 12 covers the pipeline's reach (a window entry from
// before the march start influences outputs at most 11 positions later).
// lF is updated in place: a warp reads the lF of the cells before its segment
// during its warm-up and of the three cells after it into registers, then the
// block synchronises before any warp writes lF.  lvel is read and written only
// by the warp that owns the face.
constexpr int FM_LANES = 32, FM_WARM = 12;

template <int DIR>
struct FmLine {
    const fct::Sweep<DIR> S;
    const float* Fl;    // F of the line, position 0
    const float* Vl;    // face velocity of the line
    double* lFl;
    double* lvell;
    int gs, n, c0, c1;  // stride along the line; the warp's segment [c0, c1]
    bool live;          // the lane has a line
    bool staged;        // Fl, Vl point to the line's copy in shared memory
    double vold, dt, iK4, hq, K1, dvfac;
    // forward windows (FP32), positions relative to the iteration's c
    float F5, V5, lo5;              // F, V and the low-order flux at position c+5
    float A2, A3, A4, A5;           // antidiffusive flux of faces c+2 .. c+5
    float T1, T2, T3, T4;           // Ftd of cells c+1 .. c+4
    float TM1, TM2, TM3, TM4;       // stage-1 flux term of cells c+1 .. c+4
    unsigned in1;                   // bit q-1: stage 1 of cell c+q was not clamped
    float dv3, dv4, rdv3, rdv4;     // dv and RN(1/dv) of cells c+3, c+4
    float rp2, rm2, rp3, rm3;       // ratios of cells c+2, c+3
    float C3;                       // limiter of face c+3
    // reverse windows (FP64)
    double lX2;                     // adjoint of X (stage 4) of cell c+2
    double LRP2, LRM2;              // adjoint of rp, rm of cell c+2 (face c+2 routed)
    double LT1, LT2;                // adjoint of Ftd of cells c+1, c+2 (partial)
    double LA1, LA2;                // adjoint of A of faces c+1, c+2 (partial)
    double LD1, LD2;                // adjoint of dv of cells c+1, c+2 (partial)
    double ID1, ID2;                // 1/dv of cells c+1, c+2
    double ldv0, lterm0;            // final adjoints of dv and of the stage-1 sum of cell c
    double LF0;                     // adjoint of the input F of cell c (face c added)
    double tail[3];                 // lF of cells c1+1 .. c1+3
    float F0;                       // F of cell c
    // the global loads of the next iteration, issued one iteration early
    float pF6, pV6, pF1, pV1;       // F, V at position c+6; F, V at position c+1
    double plf, plv;                // lF of cell c+3 (stage 4), lvel of face c+1

    __device__ FmLine(const Geom& g) : S(g) {}

    // F and V of the line: from shared memory when staged (Fl, Vl point
    // there, stride 1), else from global memory (read-only path)
    __device__ __forceinline__ float ldF(int q) const {
        if (!(q >= 0 && q <= n + 1)) return 0.0f;
        return staged ? Fl[q] : __ldg(Fl + q * gs);
    }
    __device__ __forceinline__ float ldV(int f) const {
        if (!(f >= 1 && f <= n + 1)) return 0.0f;
        return staged ? Vl[f] : __ldg(Vl + f * gs);
    }
    __device__ __forceinline__ bool owned(int q) const { return live && q >= c0 && q <= c1; }
    // lF of cell e as stage 4 reads it: own and earlier cells from memory, the
    // three after the segment from the registers loaded before the block barrier
    __device__ __forceinline__ double lf_at(int e) const {
        if (!live || e < 1 || e > n || e > c1 + 3) return 0.0;
        return e <= c1 ? lFl[e * gs] : (e == c1 + 1 ? tail[0] : (e == c1 + 2 ? tail[1] : tail[2]));
    }
    __device__ __forceinline__ void prefetch(int c) {
        pF6 = ldF(c + 6);
        pV6 = ldV(c + 6);
        pF1 = ldF(c + 1);
        pV1 = ldV(c + 1);
        plf = lf_at(c + 3);
        plv = owned(c + 1) && c + 1 >= 1 ? lvell[(c + 1) * gs] : 0.0;
    }

    __device__ void init(int cs) {
        F5 = ldF(cs + 5);
        V5 = ldV(cs + 5);
        lo5 = 0.0f;
        if (cs + 5 >= 1 && cs + 5 <= n + 1) {
            float a;
            fct::flux(V5, ldF(cs + 4), F5, S.dt, lo5, a);
        }
        A2 = A3 = A4 = A5 = 0.0f;
        T1 = T2 = T3 = T4 = 0.0f;
        TM1 = TM2 = TM3 = TM4 = 0.0f;
        in1 = 0u;
        dv3 = dv4 = rdv3 = rdv4 = 1.0f;
        rp2 = rm2 = rp3 = rm3 = 0.0f;
        C3 = 0.0f;
        lX2 = LRP2 = LRM2 = LT1 = LT2 = LA1 = LA2 = LD1 = LD2 = ID1 = ID2 = 0.0;
        ldv0 = lterm0 = LF0 = 0.0;
        tail[0] = tail[1] = tail[2] = 0.0;
        F0 = ldF(cs);
    }

    __device__ void load_tail() {
        for (int q = 0; q < 3; ++q) {
            const int e = c1 + 1 + q;
            tail[q] = (live && e >= 1 && e <= n) ? lFl[e * gs] : 0.0;
        }
    }

    // One iteration; the caller has issued prefetch(c).
    __device__ __forceinline__ void step(int c) {
        const float V6 = pV6, F6 = pF6, Fc1 = pF1, Vc1 = pV1;
        const double lf3 = plf, lv1 = plv;
        prefetch(c + 1);
        // s1: face c+6, cell c+5
        float lo6 = 0.0f, A6 = 0.0f;
        if (c + 6 >= 1 && c + 6 <= n + 1) fct::flux(V6, F5, F6, S.dt, lo6, A6);
        float T5 = 0.0f, TM5 = 0.0f, dv5 = 1.0f, rdv5 = 1.0f;
        bool I5 = false;
        if (c + 5 >= 1 && c + 5 <= n) {
            dv5 = S.dv(V5, V6);
            rdv5 = __frcp_rn(dv5);
            TM5 = S.term(lo5, lo6);
            const float o = div_rn_pre((F5 + TM5) * S.vol, dv5, rdv5);  // fct::ftd_from
            I5 = !(o > 1.0f || o < 0.0f);
            T5 = I5 ? o : clamp01f(o);
        }
        // s2: cell c+4
        float rp4 = 0.0f, rm4 = 0.0f;
        if (c + 4 >= 1 && c + 4 <= n) fct::limiter(S, T3, T4, T5, A4, A5, rp4, rm4);
        // s3: face c+4 (face 1's limiter is never written: 0)
        const float C4 = (c + 4 >= 2 && c + 4 <= n + 1) ? fct::face_limit(A4, rp3, rm3, rp4, rm4) : 0.0f;
        // s4: cell c+3
        double lX3 = 0.0, LD3 = 0.0, LT3 = 0.0, ID3 = 0.0;
        const int e3 = c + 3;
        if (e3 >= 1 && e3 <= n) {
            const float out = fct::stage4(S, T3, A3, C3, A4, C4, dv3, rdv3);
            const double g4 = (out >= 0.0f && out <= 1.0f) ? lf3 : 0.0;
            ID3 = rcp64((double)dv3);
            const double X = ((double)A4 * C4 - (double)A3 * C3) * iK4;
            lX3 = -g4 * vold * ID3;
            LD3 = g4 * X * vold * ID3 * ID3;
            LT3 = g4;
        }
        // s5: face c+3 (lX of cells outside 1 .. n is 0)
        double LRP3 = 0.0, LRM3 = 0.0, LA3 = 0.0;
        if (c + 3 >= 1 && c + 3 <= n + 1) {
            LA3 = (lX2 - lX3) * (double)C3 * iK4;
            if (c + 3 >= 2) {
                const double lC = (lX2 - lX3) * (double)A3 * iK4;
                if (A3 >= 0.0f) {
                    if (rp3 <= rm2) LRP3 += lC;
                    else LRM2 += lC;
                } else {
                    if (rp2 <= rm3) LRP2 += lC;
                    else LRM3 += lC;
                }
            }
        }
        // s6: cell c+2 (its lrp, lrm are complete)
        if (c + 2 >= 1 && c + 2 <= n) {
            const float a0 = A2, a1 = A3;
            const float pp = fmaxf(0.0f, a0) - fminf(0.0f, a1);
            const float pm = fmaxf(0.0f, a1) - fminf(0.0f, a0);
            const float fc = T2, fl = T1, fh = T3;
            // rp = fminf(1, RN(qp/pp)) follows qp/pp exactly when RN(qp/pp) < 1,
            // i.e. qp < pp (1 - 2^-25) (exact in FP64): no division needed
            double lqp = 0.0, lqm = 0.0, dpp = 0.0, dpm = 0.0;
            if (LRP2 != 0.0) {
                const float qp = (fmaxf(fc, fmaxf(fl, fh)) - fc) * S.hq;
                if (pp > 0.0f && (double)qp < (double)pp * (1.0 - 0x1p-25)) {
                    const double ip = rcp64((double)pp);
                    lqp = LRP2 * ip;
                    dpp = -lqp * (double)qp * ip;
                }
            }
            if (LRM2 != 0.0) {
                const float qm = (fc - fminf(fc, fminf(fl, fh))) * S.hq;
                if (pm > 0.0f && (double)qm < (double)pm * (1.0 - 0x1p-25)) {
                    const double ip = rcp64((double)pm);
                    lqm = LRM2 * ip;
                    dpm = -lqm * (double)qm * ip;
                }
            }
            // the extrema: the cell each one returned (the first argument on a tie)
            const int in_mx = (fl >= fh) ? 0 : 2;
            const int smx = (fc >= (in_mx == 0 ? fl : fh)) ? 1 : in_mx;
            const int in_mn = (fl <= fh) ? 0 : 2;
            const int smn = (fc <= (in_mn == 0 ? fl : fh)) ? 1 : in_mn;
            const double lmx = lqp * hq, lmn = -lqm * hq;
            LT2 += -lqp * hq + lqm * hq;
            // ghosts (cells 0, n+1) take no extremum adjoint
            if (smx == 0) { if (c + 1 >= 1) LT1 += lmx; }
            else if (smx == 1) LT2 += lmx;
            else if (c + 3 <= n) LT3 += lmx;
            if (smn == 0) { if (c + 1 >= 1) LT1 += lmn; }
            else if (smn == 1) LT2 += lmn;
            else if (c + 3 <= n) LT3 += lmn;
            // pp, pm of this cell depend on A of its lower (a0) and upper (a1) face
            LA2 += (a0 > 0.0f ? dpp : 0.0) - (a0 < 0.0f ? dpm : 0.0);
            LA3 += -(a1 < 0.0f ? dpp : 0.0) + (a1 > 0.0f ? dpm : 0.0);
        }
        // s7: cell c+1 (the adjoint of its Ftd is complete)
        double lterm1 = 0.0, ldv1 = 0.0, LF1 = 0.0;
        if (c + 1 >= 1 && c + 1 <= n) {
            const double h = (in1 & 1u) ? LT1 : 0.0;
            lterm1 = h * vold * ID1;
            ldv1 = LD1 - h * ((double)Fc1 + (double)TM1) * vold * ID1 * ID1;
            LF1 = lterm1;
        } else if (owned(c + 1)) {  // ghost cell: the sweep leaves it, its adjoint passes through
            LF1 = lFl[(c + 1) * gs];
        }
        // s8: face c+1
        if (c + 1 >= 1 && c + 1 <= n + 1) {
            const double l_LF = K1 * (lterm1 - lterm0);
            const double l_A = LA1;
            const float uf = Vc1, Fc0 = F0;
            const float Fh = (uf <= 0.0f) ? Fc0 : Fc1;
            const float Flo = (uf >= 0.0f) ? Fc0 : Fc1;
            if (owned(c + 1))
                lvell[(c + 1) * gs] = lv1 + (l_LF * dt * (double)Flo + l_A * dt * ((double)Fh - (double)Flo) +
                                             dvfac * (ldv1 - ldv0));
            const double w = (double)uf * dt;
            if (uf < 0.0f) LF1 += l_LF * w;  // upper cell of the face
            LF1 += l_A * w * ((uf > 0.0f ? 1.0 : 0.0) - (uf < 0.0f ? 1.0 : 0.0));
            if (uf >= 0.0f) LF0 += l_LF * w;  // lower cell
            LF0 += l_A * w * ((uf <= 0.0f ? 1.0 : 0.0) - (uf >= 0.0f ? 1.0 : 0.0));
        }
        // s9: cell c
        if (owned(c)) lFl[c * gs] = LF0;
        // shift the windows by one position
        F0 = Fc1;
        F5 = F6;
        V5 = V6;
        lo5 = lo6;
        A2 = A3; A3 = A4; A4 = A5; A5 = A6;
        T1 = T2; T2 = T3; T3 = T4; T4 = T5;
        TM1 = TM2; TM2 = TM3; TM3 = TM4; TM4 = TM5;
        in1 = (in1 >> 1) | (I5 ? 8u : 0u);
        dv3 = dv4; dv4 = dv5; rdv3 = rdv4; rdv4 = rdv5;
        rp2 = rp3; rm2 = rm3; rp3 = rp4; rm3 = rm4;
        C3 = C4;
        lX2 = lX3;
        LRP2 = LRP3; LRM2 = LRM3;
        LT1 = LT2; LT2 = LT3;
        LA1 = LA2; LA2 = LA3;
        LD1 = LD2; LD2 = LD3;
        ID1 = ID2; ID2 = ID3;
        ldv0 = ldv1;
        lterm0 = lterm1;
        LF0 = LF1;
    }
};

#ifndef VOF_FM_MINB
#define VOF_FM_MINB 4
#endif
#ifndef VOF_FM_MINB_X
#define VOF_FM_MINB_X 1
#endif
// STAGE (x lines): the block's F and V lines are first copied into shared
// memory with coalesced row loads, [line][position] with an odd pitch; the
// march then reads them there instead of 32 strided rows per warp load.
template <int DIR, int WARPS, bool STAGE>
__global__ void __launch_bounds__(FM_LANES * WARPS, DIR == 0 ? VOF_FM_MINB_X : VOF_FM_MINB)
    k_fct_adjoint_march(Geom g, const float* __restrict__ Fg, const float* __restrict__ velg, double* lFg,
                        double* __restrict__ lvelg) {
    extern __shared__ __align__(16) float fm_line_smem[];
    FmLine<DIR> L(g);
    const int n = L.S.n;
    // lines (a, b) numbered a fastest over both cross axes, one per lane, so
    // that no lane idles at the end of a row of lines
    const int na = DIR == 0 ? g.ny : g.nx, nb = DIR == 2 ? g.ny : g.nz;
    const int lane = threadIdx.x, warp = threadIdx.y;
    int line = blockIdx.x * FM_LANES + lane;
    L.live = line < na * nb;
    if (!L.live) line = na * nb - 1;  // a valid line to read; nothing is written
    const int a = 1 + line % na, b = 1 + line / na;
    const int base = DIR == 0 ? gidx(g, 0, a, b) : (DIR == 1 ? gidx(g, a, 0, b) : gidx(g, a, b, 0));
    L.gs = DIR == 0 ? 1 : (DIR == 1 ? g.px : g.plane);
    L.n = n;
    L.Fl = Fg + base;
    L.Vl = velg + base;
    L.staged = false;
    if (STAGE) {
        const int P = (n + 2) | 1;
        float* sF = fm_line_smem;
        float* sV = fm_line_smem + FM_LANES * P;
        for (int l = warp; l < FM_LANES; l += WARPS) {
            int ln = blockIdx.x * FM_LANES + l;
            if (ln >= na * nb) ln = na * nb - 1;
            const int rb = gidx(g, 0, 1 + ln % na, 1 + ln / na);  // x lines: the row (j, k)
            for (int q = lane; q < n + 2; q += FM_LANES) {
                sF[l * P + q] = __ldg(Fg + rb + q);
                sV[l * P + q] = __ldg(velg + rb + q);
            }
        }
        __syncthreads();
        L.Fl = sF + lane * P;
        L.Vl = sV + lane * P;
        L.staged = true;
    }
    L.lFl = lFg + base;
    L.lvell = lvelg + base;
    const int seg = (n + 2 + WARPS - 1) / WARPS;
    L.c0 = warp * seg;
    L.c1 = min(n + 1, L.c0 + seg - 1);
    const float vol = g.dx * g.dy * g.dz;
    L.vold = (double)vol;
    L.dt = (double)g.dt;
    L.iK4 = 1.0 / (double)L.S.h4;
    L.hq = (double)L.S.hq;
    L.K1 = DIR == 0 ? (double)g.dy * g.dz / L.vold
                    : (DIR == 1 ? (double)g.dy / ((double)g.dx * g.dy) : (double)g.dy * g.dx / L.vold);
    L.dvfac = (double)L.S.dvfac;
    // (iterations before -6 see no position of the line)
    const int cs = max(L.c0 - FM_WARM, -6);
    L.init(cs);
    L.load_tail();
    L.prefetch(cs);
    for (int c = cs; c < L.c0; ++c) L.step(c);
    __syncthreads();  // every warp has read the lF it needs from its neighbours
    for (int c = L.c0; c <= L.c1; ++c) L.step(c);
}

// ---- boundary copies, reversed ---------------------------------------------------
__global__ void k_adj_bcF_z(Geom g, double* __restrict__ l) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.nx + 1 || j > g.ny + 1) return;
    const int a = gidx(g, i, j, 0), b = gidx(g, i, j, 1), c = gidx(g, i, j, g.nz), d = gidx(g, i, j, g.nz + 1);
    l[b] += l[a];
    l[a] = 0.0;
    l[c] += l[d];
    l[d] = 0.0;
}
__global__ void k_adj_bcF_x(Geom g, double* __restrict__ l) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    if (j > g.ny + 1 || k > g.nz + 1) return;
    const int a = gidx(g, 0, j, k), b = gidx(g, 1, j, k), c = gidx(g, g.nx, j, k), d = gidx(g, g.nx + 1, j, k);
    if (g.nx < 2) {  // b == c
        l[b] += l[a];
        l[a] = 0.0;
        l[c] += l[d];
        l[d] = 0.0;
        return;
    }
    const double la = l[a], lb = l[b], lc = l[c], ld = l[d];
    l[b] = lb + la;
    l[a] = 0.0;
    l[c] = lc + ld;
    l[d] = 0.0;
}
__global__ void k_adj_bcF_y(Geom g, double* __restrict__ l) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.nx + 1 || k > g.nz + 1) return;
    const int a = gidx(g, i, 0, k), b = gidx(g, i, 1, k), c = gidx(g, i, g.ny, k), d = gidx(g, i, g.ny + 1, k);
    l[b] += l[a];
    l[a] = 0.0;
    l[c] += l[d];
    l[d] = 0.0;
}

__device__ __forceinline__ void mv(double* l, int dst, int src) {
    l[src] += l[dst];
    l[dst] = 0.0;
}
// set_bc_vel_k: u, v copied into the k ghosts, w zero at k = 1 and nz + 1.
__global__ void k_adj_bcv_z(Geom g, double* __restrict__ lu, double* __restrict__ lv, double* __restrict__ lw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.nx + 1 || j > g.ny + 1) return;
    const int k0 = gidx(g, i, j, 0), k1 = gidx(g, i, j, 1), kn = gidx(g, i, j, g.nz), kf = gidx(g, i, j, g.nz + 1);
    mv(lu, k0, k1);
    mv(lv, k0, k1);
    lw[k1] = 0.0;
    mv(lu, kf, kn);
    mv(lv, kf, kn);
    lw[kf] = 0.0;
}
// set_bc_vel_i: u zero at i = 1 and nx + 1, v, w copied into the i ghosts.
// (Its rows are strided in memory: all loads are issued before the stores.)
__global__ void k_adj_bcv_x(Geom g, double* __restrict__ lu, double* __restrict__ lv, double* __restrict__ lw) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    if (j > g.ny + 1 || k > g.nz + 1) return;
    const int i0 = gidx(g, 0, j, k), i1 = gidx(g, 1, j, k), in = gidx(g, g.nx, j, k), ir = gidx(g, g.nx + 1, j, k);
    if (g.nx < 2) {  // i = 1 is also i = nx
        lu[i1] = 0.0;
        mv(lv, i0, i1);
        mv(lw, i0, i1);
        lu[ir] = 0.0;
        mv(lv, ir, in);
        mv(lw, ir, in);
        return;
    }
    const double v0 = lv[i0], v1 = lv[i1], vn = lv[in], vr = lv[ir];
    const double w0 = lw[i0], w1 = lw[i1], wn = lw[in], wr = lw[ir];
    lu[i1] = 0.0;
    lu[ir] = 0.0;
    lv[i1] = v1 + v0;
    lv[i0] = 0.0;
    lw[i1] = w1 + w0;
    lw[i0] = 0.0;
    lv[in] = vn + vr;
    lv[ir] = 0.0;
    lw[in] = wn + wr;
    lw[ir] = 0.0;
}
// set_bc_vel_j: v zero at j = 1 and ny + 1, u, w copied into the j ghosts.
__global__ void k_adj_bcv_y(Geom g, double* __restrict__ lu, double* __restrict__ lv, double* __restrict__ lw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.nx + 1 || k > g.nz + 1) return;
    const int j0 = gidx(g, i, 0, k), j1 = gidx(g, i, 1, k), jn = gidx(g, i, g.ny, k), jt = gidx(g, i, g.ny + 1, k);
    mv(lu, j0, j1);
    lv[j1] = 0.0;
    mv(lw, j0, j1);
    mv(lu, jt, jn);
    lv[jt] = 0.0;
    mv(lw, jt, jn);
}

// Wall flags of a cell (i==1, i==nx, j==1, j==ny, k==1, k==nz; bits 0..5) and
// -N mu of the transposed Jacobi sweep (below) at cell c.
__device__ __forceinline__ int wall_flags(const Geom& g, int i, int j, int k) {
    return (i == 1) | ((i == g.nx) << 1) | ((j == 1) << 2) | ((j == g.ny) << 3) | ((k == 1) << 4) |
           ((k == g.nz) << 5);
}
__device__ __forceinline__ double neg_N(const Geom& g, const double* mu, int c, int i, int j, int k) {
    const double cxx = (double)(g.dxi * g.dxi), cyy = (double)(g.dyi * g.dyi), czz = (double)(g.dzi * g.dzi);
    double s = 0.0;
    if (i != g.nx) s += cxx * mu[c + 1];
    if (i != 1) s += cxx * mu[c - 1];
    if (j != g.ny) s += cyy * mu[c + g.px];
    if (j != 1) s += cyy * mu[c - g.px];
    if (k != g.nz) s += czz * mu[c + g.plane];
    if (k != 1) s += czz * mu[c - g.plane];
    return -s;
}
// ---- velocity correction, reversed (gather over the six faces of a cell) -----------
// Face q along axis a (its cells q - st and q): u_q = u*_q - dt/r (p_q - p_{q-st}) h^-1,
// r = (rho_q + rho_{q-st}) / 2.  Cell c collects, from its lower faces (q = c)
// and upper faces (q = c + st), the adjoints of p_c and rho_c.  The face
// adjoint itself becomes the adjoint of u*, v*, w* at that face: the advection
// kernel reads it from lu, lv, lw and accumulates the adjoint of the step's
// start velocity into a cleared second set of fields (the correction wrote
// every face, so nothing else of lu, lv, lw carries over), and the two sets
// swap.
//
// FUSE (plain step with Jacobi sweeps): the cell's pressure adjoint is -N mu_prev
// (the last transposed Jacobi stage of the later step, deferred to here while
// `pending`; N and the stages are those of k_adj_jacobi) or lp[c], plus the
// correction's contribution; the first transposed stage follows at once:
// mu0 = that / ap into mu_out, lrhs = mu0 -- the same operations, in the same
// order, as the separate stage kernels.  Otherwise lp[c] += the contribution.
template <bool FUSE>
__global__ void __launch_bounds__(256) k_adj_update(Geom g, Range R, const float* __restrict__ F,
                                                    const float* __restrict__ p, const double* __restrict__ lu,
                                                    const double* __restrict__ lv, const double* __restrict__ lw,
                                                    double* __restrict__ lp, double* __restrict__ lrho,
                                                    int pending, InvAp ia, double* __restrict__ mu_out,
                                                    double* __restrict__ lrhs) {
    RANGE_CELL(R);
    const int c = gidx(g, i, j, k);
    const int pos[3] = {i, j, k}, len[3] = {g.nx, g.ny, g.nz}, st[3] = {1, g.px, g.plane};
    const double hinv[3] = {(double)g.dxi, (double)g.dyi, (double)g.dzi};
    const double* lvel[3] = {lu, lv, lw};
    const float rho_c = rho_of(g, F[c]);
    const double dt = (double)g.dt, pc = (double)p[c];
    double lpc = 0.0, lrc = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (pos[a] >= 2) {  // lower face: c is its upper cell
            const int m = c - st[a];
            const double gv = lvel[a][c];
            if (gv != 0.0) {
                const double ir = rcp64((double)(0.5f * (rho_c + rho_of(g, F[m]))));
                lpc -= gv * dt * ir * hinv[a];
                lrc += 0.5 * gv * dt * (pc - (double)p[m]) * hinv[a] * ir * ir;
            }
        }
        if (pos[a] + 1 <= len[a]) {  // upper face: c is its lower cell
            const int q = c + st[a];
            const double gv = lvel[a][q];
            if (gv != 0.0) {
                const double ir = rcp64((double)(0.5f * (rho_of(g, F[q]) + rho_c)));
                lpc += gv * dt * ir * hinv[a];
                lrc += 0.5 * gv * dt * ((double)p[q] - pc) * hinv[a] * ir * ir;
            }
        }
    }
    if (FUSE) {
        const double lpf = (pending ? neg_N(g, lp, c, i, j, k) : lp[c]) + lpc;
        const double mu = lpf * ia.v[wall_flags(g, i, j, k)];
        mu_out[c] = mu;
        lrhs[c] = mu;
    } else {
        lp[c] += lpc;
    }
    lrho[c] = lrc;
}

// ---- Jacobi, transposed, on mu = lambda / ap --------------------------------------
// Forward sweep: p' = (rhs - N p) / ap.  Reverse: mu_k = lambda_k / ap,
// lrhs += mu_k, lambda_{k-1} = -N mu_k; carried as mu: mu_{k-1} = -N mu_k / ap.
// inv_ap[flags] = 1 / ap (FP32 ap of the forward, in its order) for the six
// wall flags (i==1, i==nx, j==1, j==ny, k==1, k==nz) of a cell.
// mode 0: mu = lin / ap, lrhs = mu;  1: mu = -N lin / ap, lrhs += mu;  2: out = -N lin.
__global__ void __launch_bounds__(256) k_adj_jacobi(Geom g, Range R, InvAp ia, const double* __restrict__ lin,
                                                    double* __restrict__ lout, double* __restrict__ lrhs, int mode) {
    RANGE_CELL(R);
    const int c = gidx(g, i, j, k);
    if (mode == 2) {
        lout[c] = neg_N(g, lin, c, i, j, k);
        return;
    }
    const double inv = ia.v[wall_flags(g, i, j, k)];
    const double mu = (mode == 0 ? lin[c] : neg_N(g, lin, c, i, j, k)) * inv;
    lout[c] = mu;
    lrhs[c] = mode == 0 ? mu : lrhs[c] + mu;
}

// Two consecutive transposed sweeps in one pass (modes as k_adj_jacobi: A is 0
// or 1, B is 1 or 2): stage A on lin gives mu_a, stage B on mu_a gives the
// output; lrhs takes mu_a (A == 0: lrhs = mu_a, else lrhs += mu_a) and then
// mu_b (B == 1).  A block owns a 32 x 8 column tile and a chunk of planes and
// marches up in k with plane rings in shared memory: lin with a two-cell
// in-plane halo, mu_a with a one-cell halo (computed redundantly at the tile
// edge), so HBM sees lin, lrhs and the output once per two sweeps.
constexpr int AJ_TX = 32, AJ_TY = 8, AJ_T = AJ_TX * AJ_TY;
constexpr int AJ_NIN = (AJ_TY + 4) * (AJ_TX + 4), AJ_NA = (AJ_TY + 2) * (AJ_TX + 2);
// A point of a plane tile with its in-plane geometry: shared index, global
// in-plane offset, wall flags (bits 0..3 of wall_flags) and whether it is a cell.
struct AjPoint {
    int sidx, off, flags;
    bool cell;
};
__device__ __forceinline__ AjPoint aj_point(const Geom& g, int q, int w, int h, int i0, int j0) {
    const int y = q / w, x = q % w;
    const int i = i0 - h + x, j = j0 - h + y;
    AjPoint p;
    p.sidx = q;
    p.cell = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny;
    p.off = p.cell ? gidx(g, i, j, 0) : 0;
    p.flags = (i == 1) | ((i == g.nx) << 1) | ((j == 1) << 2) | ((j == g.ny) << 3);
    return p;
}
// -N at a point of a ring of planes (row width w) from its in-plane flags and k
__device__ __forceinline__ double aj_negN(const double* pc, const double* pm, const double* pp, int q, int w,
                                          int flags, int k, int nz, double cxx, double cyy, double czz) {
    double s = 0.0;
    if (!(flags & 2)) s += cxx * pc[q + 1];
    if (!(flags & 1)) s += cxx * pc[q - 1];
    if (!(flags & 8)) s += cyy * pc[q + w];
    if (!(flags & 4)) s += cyy * pc[q - w];
    if (k != nz) s += czz * pp[q];
    if (k != 1) s += czz * pm[q];
    return -s;
}
template <int A, int B>
__global__ void __launch_bounds__(AJ_T) k_adj_jacobi2(Geom g, InvAp ia, const double* __restrict__ lin,
                                                     double* __restrict__ lout, double* __restrict__ lrhs,
                                                     int kchunk) {
    constexpr int WI = AJ_TX + 4, WA = AJ_TX + 2;
    __shared__ double sIn[3][AJ_NIN];
    __shared__ double sA[3][AJ_NA];
    const int tid = threadIdx.y * AJ_TX + threadIdx.x;
    const int i0 = 1 + blockIdx.x * AJ_TX, j0 = 1 + blockIdx.y * AJ_TY;
    const int k0 = 1 + blockIdx.z * kchunk, k1 = min(g.nz, k0 + kchunk - 1);
    const double cxx = (double)(g.dxi * g.dxi), cyy = (double)(g.dyi * g.dyi), czz = (double)(g.dzi * g.dzi);
    const int plane = g.plane;
    // this thread's points: two of the lin tile (halo 2), two of the stage-A tile (halo 1), one output
    const AjPoint L0 = aj_point(g, tid, WI, 2, i0, j0);
    const bool has_l1 = tid + AJ_T < AJ_NIN;
    const AjPoint L1 = aj_point(g, has_l1 ? tid + AJ_T : tid, WI, 2, i0, j0);
    const AjPoint S0 = aj_point(g, tid, WA, 1, i0, j0);
    const bool has_s1 = tid + AJ_T < AJ_NA;
    const AjPoint S1 = aj_point(g, has_s1 ? tid + AJ_T : tid, WA, 1, i0, j0);
    // the stage-A point's index in the lin tile: (y + 1) * WI + x + 1
    const int S0in = (S0.sidx / WA + 1) * WI + S0.sidx % WA + 1, S1in = (S1.sidx / WA + 1) * WI + S1.sidx % WA + 1;
    const int io = i0 + (int)threadIdx.x, jo = j0 + (int)threadIdx.y;
    const bool out_ok = io <= g.nx && jo <= g.ny;
    const int oflags = (io == 1) | ((io == g.nx) << 1) | ((jo == 1) << 2) | ((jo == g.ny) << 3);
    const int ooff = out_ok ? gidx(g, io, jo, 0) : 0;
    const int oA = (threadIdx.y + 1) * WA + threadIdx.x + 1;
    auto slot = [](int k) { return (k + 3) % 3; };  // k >= -2
    auto kflags = [&](int k) { return ((k == 1) << 4) | ((k == g.nz) << 5); };
    auto ld = [&](const AjPoint& p, int k) { return (p.cell && k >= 1 && k <= g.nz) ? lin[p.off + k * plane] : 0.0; };
    // lin of the first plane in registers
    double n0 = ld(L0, k0 - 2), n1 = has_l1 ? ld(L1, k0 - 2) : 0.0;
    for (int t = k0 - 3; t <= k1 + 1; ++t) {
        // lin at plane t+1 into the ring; the next plane's loads go out now
        {
            const int sl = slot(t + 1);
            sIn[sl][L0.sidx] = n0;
            if (has_l1) sIn[sl][L1.sidx] = n1;
            n0 = ld(L0, t + 2);
            if (has_l1) n1 = ld(L1, t + 2);
        }
        const int kb = t - 1;
        const bool do_b = kb >= k0 && out_ok;
        const double rhs_old = (A == 1 && do_b) ? lrhs[ooff + kb * plane] : 0.0;
        __syncthreads();
        // stage A at plane t on the tile and its one-cell halo
        if (t >= k0 - 1) {
            const int sc = slot(t);
            const double *pc = sIn[sc], *pm = sIn[slot(t - 1)], *pp = sIn[slot(t + 1)];
            const bool kin = t >= 1 && t <= g.nz;
            const int kf = kflags(t);
            {
                double v = 0.0;
                if (S0.cell && kin)
                    v = (A == 0 ? pc[S0in] : aj_negN(pc, pm, pp, S0in, WI, S0.flags, t, g.nz, cxx, cyy, czz)) *
                        ia.v[S0.flags | kf];
                sA[sc][S0.sidx] = v;
            }
            if (has_s1) {
                double v = 0.0;
                if (S1.cell && kin)
                    v = (A == 0 ? pc[S1in] : aj_negN(pc, pm, pp, S1in, WI, S1.flags, t, g.nz, cxx, cyy, czz)) *
                        ia.v[S1.flags | kf];
                sA[sc][S1.sidx] = v;
            }
        }
        __syncthreads();
        // stage B at plane t-1 on the tile
        if (do_b) {
            const int sb = slot(kb);
            const double mua = sA[sb][oA];
            const double nb = aj_negN(sA[sb], sA[slot(kb - 1)], sA[slot(kb + 1)], oA, WA, oflags, kb, g.nz, cxx, cyy,
                                      czz);
            const int c = ooff + kb * plane;
            const double r = A == 0 ? mua : rhs_old + mua;
            if (B == 1) {
                const double mub = nb * ia.v[oflags | kflags(kb)];
                lout[c] = mub;
                lrhs[c] = r + mub;
            } else {
                lout[c] = nb;
                lrhs[c] = r;
            }
        }
    }
}

// ---- advection, reversed (scatter with FP64 atomics) --------------------------------
// One momentum component q at face c: q* = q + dt (visc + adv + g_q),
// adv = -a dq/dx - b dq/dy - cc dq/dz, upwinded by the signs of a, b, cc;
// (a, b, cc) are q itself along its own axis and 4-point averages otherwise.
template <int COMP>
__device__ __forceinline__ double adj_momentum(const Geom& g, int c, int i, int j, int k, const float* u,
                                               const float* v, const float* w, double G, double nuc, double* lu,
                                               double* lv, double* lw, double& lnu) {
    const int sx = 1, sy = g.px, sz = g.plane;
    const float* q = COMP == 0 ? u : (COMP == 1 ? v : w);
    double* lq = COMP == 0 ? lu : (COMP == 1 ? lv : lw);
    int ia[4], ib[4];
    float a, b, cc;
    double *la, *lb;
    if (COMP == 0) {
        ia[0] = c - sx; ia[1] = c - sx + sy; ia[2] = c; ia[3] = c + sy;
        ib[0] = c - sx; ib[1] = c - sx + sz; ib[2] = c; ib[3] = c + sz;
        a = q[c];
        b = 0.25f * (v[ia[0]] + v[ia[1]] + v[ia[2]] + v[ia[3]]);
        cc = 0.25f * (w[ib[0]] + w[ib[1]] + w[ib[2]] + w[ib[3]]);
        la = lv;
        lb = lw;
    } else if (COMP == 1) {
        ia[0] = c - sy; ia[1] = c; ia[2] = c + sx - sy; ia[3] = c + sx;
        ib[0] = c - sy + sz; ib[1] = c - sy; ib[2] = c; ib[3] = c + sz;
        a = 0.25f * (u[ia[0]] + u[ia[1]] + u[ia[2]] + u[ia[3]]);
        b = q[c];
        cc = 0.25f * (w[ib[0]] + w[ib[1]] + w[ib[2]] + w[ib[3]]);
        la = lu;
        lb = lw;
    } else {
        ia[0] = c + sx - sz; ia[1] = c - sz; ia[2] = c + sx; ia[3] = c;
        ib[0] = c + sy - sz; ib[1] = c - sz; ib[2] = c; ib[3] = c + sy;
        a = 0.25f * (u[ia[0]] + u[ia[1]] + u[ia[2]] + u[ia[3]]);
        b = 0.25f * (v[ib[0]] + v[ib[1]] + v[ib[2]] + v[ib[3]]);
        cc = q[c];
        la = lu;
        lb = lv;
    }
    const double hx = (double)g.dxi, hy = (double)g.dyi, hz = (double)g.dzi;
    const double hx2 = hx * hx, hy2 = hy * hy, hz2 = hz * hz;
    const double qc = q[c], qxm = q[c - sx], qxp = q[c + sx], qym = q[c - sy], qyp = q[c + sy], qzm = q[c - sz],
                 qzp = q[c + sz];
    const bool ux = a > 0.0f, uy = b > 0.0f, uz = cc > 0.0f;
    const double dqdx = ux ? (qc - qxm) * hx : (qxp - qc) * hx;
    const double dqdy = uy ? (qc - qym) * hy : (qyp - qc) * hy;
    const double dqdz = uz ? (qc - qzm) * hz : (qzp - qc) * hz;
    const double Gd = G * (double)g.dt;
    lnu += Gd * ((qxm - 2.0 * qc + qxp) * hx2 + (qym - 2.0 * qc + qyp) * hy2 + (qzm - 2.0 * qc + qzp) * hz2);
    double own = G - Gd * nuc * 2.0 * (hx2 + hy2 + hz2);
    // neighbours along each axis: viscous term, plus the upwind difference
    // on the side the forward took (one atomic per neighbour)
    const double ga = -Gd * (double)a, gb = -Gd * (double)b, gc = -Gd * (double)cc;
    const double vx = Gd * nuc * hx2, vy = Gd * nuc * hy2, vz = Gd * nuc * hz2;
    if (ux) { own += ga * hx; atomicAdd(lq + c - sx, vx + -ga * hx); atomicAdd(lq + c + sx, vx); }
    else { own -= ga * hx; atomicAdd(lq + c - sx, vx); atomicAdd(lq + c + sx, vx + ga * hx); }
    if (uy) { own += gb * hy; atomicAdd(lq + c - sy, vy + -gb * hy); atomicAdd(lq + c + sy, vy); }
    else { own -= gb * hy; atomicAdd(lq + c - sy, vy); atomicAdd(lq + c + sy, vy + gb * hy); }
    if (uz) { own += gc * hz; atomicAdd(lq + c - sz, vz + -gc * hz); atomicAdd(lq + c + sz, vz); }
    else { own -= gc * hz; atomicAdd(lq + c - sz, vz); atomicAdd(lq + c + sz, vz + gc * hz); }
    const double l_a = -Gd * dqdx, l_b = -Gd * dqdy, l_c = -Gd * dqdz;
    if (COMP == 0) {
        own += l_a;
        for (int t = 0; t < 4; ++t) { atomicAdd(la + ia[t], 0.25 * l_b); atomicAdd(lb + ib[t], 0.25 * l_c); }
    } else if (COMP == 1) {
        own += l_b;
        for (int t = 0; t < 4; ++t) { atomicAdd(la + ia[t], 0.25 * l_a); atomicAdd(lb + ib[t], 0.25 * l_c); }
    } else {
        own += l_c;
        for (int t = 0; t < 4; ++t) { atomicAdd(la + ia[t], 0.25 * l_a); atomicAdd(lb + ib[t], 0.25 * l_b); }
    }
    atomicAdd(lq + c, own);
    return Gd;
}

// The rhs (voftrial1.cu:418-422: rhs = rho/dt div(u*)) reversed first, as a
// gather over the cells sharing this cell's faces (has_rhs = 0: no Jacobi
// sweeps, no rhs adjoint): u*, v*, w* at the cell's lower faces and rho take
// lrhs of the cell and of its lower neighbours.  Then the advection of the
// three momentum components at those faces, and the adjoint of rho and nu
// (cal_nu_rho_kernel, voftrial1.cu:95-104): with lrho complete (correction
// and rhs) and lnu from the three momentum equations of this cell,
// lF[c] += (lrho drho/dF + lnu dnu/dF).  lu, lv, lw are zero on entry (the
// correction overwrote every face).  lus, lvs, lws: the adjoints of u*, v*,
// w* from the correction (the face adjoints of the corrected velocity).
// dL/dg: each block adds its sums to its own slot of `partial` (summed once
// at the end).
__global__ void __launch_bounds__(256) k_adj_advect(Geom g, Range R, const float* __restrict__ F,
                                                    const float* __restrict__ u, const float* __restrict__ v,
                                                    const float* __restrict__ w, const float* __restrict__ us,
                                                    const float* __restrict__ vs, const float* __restrict__ ws,
                                                    const double* __restrict__ lrhs, int has_rhs,
                                                    const double* __restrict__ lus, const double* __restrict__ lvs,
                                                    const double* __restrict__ lws, double* __restrict__ lu,
                                                    double* __restrict__ lv, double* __restrict__ lw,
                                                    const double* __restrict__ lrho, double* __restrict__ lF,
                                                    double* __restrict__ partial) {
    const int i = R.i0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = R.j0 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = R.k0 + blockIdx.z * blockDim.z + threadIdx.z;
    double gsum[3] = {0.0, 0.0, 0.0};
    if (i <= R.i1 && j <= R.j1 && k <= R.k1) {
        const int c = gidx(g, i, j, k);
        const float Fc = F[c];
        double Gu = lus[c], Gv = lvs[c], Gw = lws[c], lr = lrho[c];
        if (has_rhs) {
            const int sy = g.px, sz = g.plane;
            const double idt = rcp64((double)g.dt), dxi = (double)g.dxi, dyi = (double)g.dyi, dzi = (double)g.dzi;
            const double gr = lrhs[c];
            const double div = ((double)us[c + 1] - us[c]) * dxi + ((double)vs[c + sy] - vs[c]) * dyi +
                               ((double)ws[c + sz] - ws[c]) * dzi;
            lr += gr * div * idt;
            const double kk = gr * (double)rho_of(g, Fc) * idt;
            const double kx = i >= 2 ? lrhs[c - 1] * (double)rho_of(g, F[c - 1]) * idt : 0.0;
            const double ky = j >= 2 ? lrhs[c - sy] * (double)rho_of(g, F[c - sy]) * idt : 0.0;
            const double kz = k >= 2 ? lrhs[c - sz] * (double)rho_of(g, F[c - sz]) * idt : 0.0;
            Gu += (kx - kk) * dxi;
            Gv += (ky - kk) * dyi;
            Gw += (kz - kk) * dzi;
        }
        const double nuc = (double)nu_of(g, Fc);
        double lnc = 0.0;
        if (i >= 2 && Gu != 0.0) gsum[0] = adj_momentum<0>(g, c, i, j, k, u, v, w, Gu, nuc, lu, lv, lw, lnc);
        if (j >= 2 && Gv != 0.0) gsum[1] = adj_momentum<1>(g, c, i, j, k, u, v, w, Gv, nuc, lu, lv, lw, lnc);
        if (k >= 2 && Gw != 0.0) gsum[2] = adj_momentum<2>(g, c, i, j, k, u, v, w, Gw, nuc, lu, lv, lw, lnc);
        if ((lr != 0.0 || lnc != 0.0) && Fc >= 0.0f && Fc <= 1.0f)
            lF[c] += lr * ((double)g.rho_l - (double)g.rho_g) + lnc * ((double)g.nu_l - (double)g.nu_g);
    }
    // deterministic block sums of dL/dg
    __shared__ double sh[3][8];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    for (int q = 0; q < 3; ++q)
        for (int o = 16; o > 0; o >>= 1) gsum[q] += __shfl_down_sync(0xffffffffu, gsum[q], o);
    if ((tid & 31) == 0)
        for (int q = 0; q < 3; ++q) sh[q][tid >> 5] = gsum[q];
    __syncthreads();
    if (tid == 0) {
        const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        for (int q = 0; q < 3; ++q) {
            double t = 0.0;
            for (int wv = 0; wv < 8; ++wv) t += sh[q][wv];
            partial[3 * blk + q] += t;
        }
    }
}

// sums[q] += Sigma_b partial[ncomp b + q] (q < ncomp), in a fixed order:
// each of the 256 threads sums a strided subset, then thread 0 the 256 results.
__global__ void k_fold_add(const double* __restrict__ partial, int nblk, int ncomp, double* sums) {
    __shared__ double sh[3][256];
    for (int q = 0; q < ncomp; ++q) {
        double t = 0.0;
        for (int b = threadIdx.x; b < nblk; b += blockDim.x) t += partial[ncomp * b + q];
        sh[q][threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int q = 0; q < ncomp; ++q) {
            double t = 0.0;
            for (int b = 0; b < (int)blockDim.x; ++b) t += sh[q][b];
            sums[q] += t;
        }
}

// ---- the loss: L = Sigma over the box of F dV; lF = dV there ----------------------------
__device__ __forceinline__ bool in_box(const Geom& g, const double* b, int i, int j, int k) {
    const double xc = (i - 0.5) * (double)g.dx, yc = (j - 0.5) * (double)g.dy, zc = (k - 0.5) * (double)g.dz;
    return xc > b[0] && xc < b[1] && yc > b[2] && yc < b[3] && zc > b[4] && zc < b[5];
}
struct Box6 {
    double b[6];
};
__global__ void __launch_bounds__(256) k_seed(Geom g, Range R, Box6 box, const float* __restrict__ F,
                                              double* __restrict__ lF, double* __restrict__ partial) {
    const int i = R.i0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = R.j0 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = R.k0 + blockIdx.z * blockDim.z + threadIdx.z;
    const double dV = (double)g.dx * (double)g.dy * (double)g.dz;
    double acc = 0.0;
    if (i <= R.i1 && j <= R.j1 && k <= R.k1) {
        const int c = gidx(g, i, j, k);
        const bool inside = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz && in_box(g, box.b, i, j, k);
        lF[c] = inside ? dV : 0.0;
        if (inside) acc = (double)F[c] * dV;
    }
    __shared__ double sh[8];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((tid & 31) == 0) sh[tid >> 5] = acc;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int wv = 0; wv < 8; ++wv) t += sh[wv];
        partial[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = t;
    }
}

// ---- host -------------------------------------------------------------------------
inline Range axis_range(const Geom& g, int dir, int lo, int hi_extra) {
    Range r = interior(g);
    if (dir == 0) { r.i0 = lo; r.i1 = g.nx + hi_extra; }
    else if (dir == 1) { r.j0 = lo; r.j1 = g.ny + hi_extra; }
    else { r.k0 = lo; r.k1 = g.nz + hi_extra; }
    return r;
}

template <int DIR, int LPB>
cudaError_t launch_fct_adjoint(const Geom& g, const float* Fs, const float* vel, double* lF, double* lvel,
                               cudaStream_t s) {
    const int n = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
    const size_t smem = fa_smem_bytes(LPB, n);
    cudaError_t r = cudaFuncSetAttribute(k_fct_adjoint<DIR, LPB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (r != cudaSuccess) return r;
    dim3 grid;
    if (DIR == 0) grid = dim3((g.ny + LPB - 1) / LPB, g.nz);
    else if (DIR == 1) grid = dim3((g.nx + LPB - 1) / LPB, g.nz);
    else grid = dim3((g.nx + LPB - 1) / LPB, g.ny);
    k_fct_adjoint<DIR, LPB><<<grid, FA_THREADS, smem, s>>>(g, Fs, vel, lF, lvel);
    return cudaGetLastError();
}

// Largest shared memory one block may take.
size_t fa_smem_limit() {
    static size_t lim = 0;
    if (!lim) {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess)
            lim = (size_t)v;
    }
    return lim;
}

#ifndef VOF_FM_WARPS
#define VOF_FM_WARPS 4
#endif
constexpr int FM_WARPS = VOF_FM_WARPS;
template <int DIR>
cudaError_t launch_fct_adjoint_march(const Geom& g, const float* Fs, const float* vel, double* lF, double* lvel,
                                     cudaStream_t s) {
    const int na = DIR == 0 ? g.ny : g.nx;
    const int nb = DIR == 2 ? g.ny : g.nz;
    const dim3 grid((na * nb + FM_LANES - 1) / FM_LANES), blk(FM_LANES, FM_WARPS);
    const int n = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
    const size_t smem = sizeof(float) * 2 * FM_LANES * (size_t)((n + 2) | 1);
    if (DIR == 0 && smem <= fa_smem_limit()) {
        cudaError_t r = cudaFuncSetAttribute(k_fct_adjoint_march<DIR, FM_WARPS, true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (r != cudaSuccess) return r;
        k_fct_adjoint_march<DIR, FM_WARPS, true><<<grid, blk, smem, s>>>(g, Fs, vel, lF, lvel);
    } else {
        k_fct_adjoint_march<DIR, FM_WARPS, false><<<grid, blk, 0, s>>>(g, Fs, vel, lF, lvel);
    }
    return cudaGetLastError();
}

// The line march runs one lane per grid line: it needs enough lines to fill
// the GPU; smaller grids take the shared-memory kernel (threads along lines).
constexpr long FM_MIN_LINES = 16384;
template <int DIR>
cudaError_t sweep_adjoint(AdjEngine& e, const float* Fs, const float* vel, double* lvel, cudaStream_t s) {
    const Geom& g = e.g;
    const long lines = DIR == 0 ? (long)g.ny * g.nz : (DIR == 1 ? (long)g.nx * g.nz : (long)g.nx * g.ny);
    if (e.fct_march == 2 || (e.fct_march && lines >= FM_MIN_LINES))
        return launch_fct_adjoint_march<DIR>(g, Fs, vel, e.lF, lvel, s);
    {  // one fused kernel when a block of lines fits in shared memory
        const int n = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
        // the most lines per block with at least two blocks per SM, else the most that fit
        const size_t lim = fa_smem_limit(), two = lim / 2 - 1024;
        if (fa_smem_bytes(8, n) <= two) return launch_fct_adjoint<DIR, 8>(g, Fs, vel, e.lF, lvel, s);
        if (fa_smem_bytes(4, n) <= two) return launch_fct_adjoint<DIR, 4>(g, Fs, vel, e.lF, lvel, s);
        if (fa_smem_bytes(2, n) <= two) return launch_fct_adjoint<DIR, 2>(g, Fs, vel, e.lF, lvel, s);
        if (fa_smem_bytes(2, n) <= lim) return launch_fct_adjoint<DIR, 2>(g, Fs, vel, e.lF, lvel, s);
    }
    const Range I = interior(g);
    const dim3 gi = grid_of(I);
    k_fs1<DIR><<<gi, kBlk, 0, s>>>(g, I, Fs, vel, e.Ftd);
    k_fs2<DIR><<<gi, kBlk, 0, s>>>(g, I, Fs, vel, e.Ftd, e.A, e.rp, e.rm);
    k_fs3<DIR><<<gi, kBlk, 0, s>>>(g, I, e.A, e.rp, e.rm, e.C);
    k_as4<DIR><<<gi, kBlk, 0, s>>>(g, I, vel, e.Ftd, e.A, e.C, e.lF, e.lX, e.ldv, e.lown);
    k_as3<DIR><<<gi, kBlk, 0, s>>>(g, I, e.Ftd, e.A, e.rp, e.rm, e.lX, e.lmx, e.lmn, e.lpp, e.lpm, e.lown, e.sel);
    k_as2<DIR><<<gi, kBlk, 0, s>>>(g, I, Fs, vel, e.lmx, e.lmn, e.sel, e.lown, e.ldv, e.lterm);
    const Range Rf = axis_range(g, DIR, 1, 1);
    k_as1<DIR><<<grid_of(Rf), kBlk, 0, s>>>(g, Rf, Fs, vel, e.A, e.C, e.lX, e.lpp, e.lpm, e.ldv, e.lterm, e.lLF,
                                             e.lA, lvel);
    const Range Rc = axis_range(g, DIR, 0, 1);
    k_as0<DIR><<<grid_of(Rc), kBlk, 0, s>>>(g, Rc, vel, e.lterm, e.lLF, e.lA, e.lF);
    return cudaGetLastError();
}

cudaError_t copy_field(float* dst, const float* src, size_t elems, cudaStream_t s) {
    return cudaMemcpyAsync(dst, src, elems * sizeof(float), cudaMemcpyDeviceToDevice, s);
}

cudaError_t load_state(AdjEngine& e, const AdjState& x, cudaStream_t s) {
    float* dst[5] = {e.wb.F, e.wb.u, e.wb.v, e.wb.w, e.wb.p0};
    cudaError_t r;
    for (int q = 0; q < 5; ++q)
        if ((r = copy_field(dst[q], x.f[q], e.elems, s)) != cudaSuccess) return r;
    if (e.conv)
        return cudaMemcpyAsync(e.p64, x.p64, e.elems * sizeof(double), cudaMemcpyDeviceToDevice, s);
    return cudaSuccess;
}

// The pressure of the step whose predictor and rhs are in e.wb: the plain
// Jacobi sweeps, or the convergent solve warm-started from e.p64 (the same
// call the forward made, so the same bits).  Returns the FP32 pressure.
cudaError_t step_pressure(AdjEngine& e, const float** pafter, cudaStream_t s) {
    if (e.conv) {
        cudaError_t r = mg_solve(e.g, e.mg_fwd, e.wb.rhs, e.p64, e.wb.p0, e.tol, e.max_outer, nullptr, s, e.cap);
        *pafter = e.wb.p0;
        return r == cudaErrorNotReady ? cudaSuccess : r;  // the forward took the same unconverged iterate
    }
    int par = 0;
    cudaError_t r = plain_pressure(e.g, e.wb, e.jacobi_iters, &par, s);
    *pafter = par ? e.wb.p1 : e.wb.p0;
    return r;
}

// Sweep axes of step istep, in order (voftrial1.cu:1384-1396).
inline const int* sweep_order(int istep) {
    static const int order[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
    return order[((istep % 3) + 3) % 3];
}

// What a reversed step reads: the start state, the predictor's output, the
// pressure after the solve, the corrected velocity and each sweep's input F.
struct StepData {
    const float *F, *u, *v, *w;
    const float *us, *vs, *ws;
    const float* p;
    const float* vel[3];
    const float* Fsw[3];
};

// The intermediates of step istep recomputed from its start state x with the
// engine's buffers (the forward's kernels, so the forward's bits).
cudaError_t recompute_step(AdjEngine& e, const AdjState& x, int istep, StepData* d, cudaStream_t s) {
    const Geom& g = e.g;
    cudaError_t r;
    if ((r = load_state(e, x, s)) != cudaSuccess) return r;
    if ((r = plain_front(g, e.wb, s)) != cudaSuccess) return r;
    const float* pafter = nullptr;
    if ((r = step_pressure(e, &pafter, s)) != cudaSuccess) return r;
    if ((r = plain_correct(g, e.wb, pafter, s)) != cudaSuccess) return r;
    const int* dirs = sweep_order(istep);
    const float* velof[3] = {e.wb.u, e.wb.v, e.wb.w};
    if ((r = copy_field(e.Fin1, x.f[0], e.elems, s)) != cudaSuccess ||
        (r = fct_launch(g, dirs[0], false, e.Fin1, velof[dirs[0]], s)) != cudaSuccess ||
        (r = copy_field(e.Fin2, e.Fin1, e.elems, s)) != cudaSuccess ||
        (r = fct_launch(g, dirs[1], false, e.Fin2, velof[dirs[1]], s)) != cudaSuccess)
        return r;
    *d = StepData{x.f[0], x.f[1], x.f[2], x.f[3], e.wb.us, e.wb.vs, e.wb.ws, pafter,
                  {velof[0], velof[1], velof[2]}, {x.f[0], e.Fin1, e.Fin2}};
    return cudaSuccess;
}

// One step of the segment replay on the engine's buffers, keeping its
// intermediates in mid: the predictor writes mid's u*, v*, w*; the sweeps run
// out of place, Fin -> mid's F after the first sweep -> mid's F after the
// second -> Fout.  The start velocity is read from vin, the corrected velocity
// written to vout (which may be vin).  *par: the Jacobi ping-pong parity of
// the plain step; *pafter: the pressure after the solve.  (mid's F buffers
// were cleared at allocation: their ghost cells, which the sweeps do not
// write, enter the next sweep only through zero wall velocities.)
cudaError_t replay_step_keep(AdjEngine& e, int istep, const AdjMid& mid, const float* Fin, float* Fout,
                             float* const vin[3], float* const vout[3], int* par, const float** pafter,
                             cudaStream_t s) {
    const Geom& g = e.g;
    PlainBuffers b = e.wb;
    b.F = const_cast<float*>(Fin);  // read only by the predictor, rhs and correction
    b.us = mid.f[0];
    b.vs = mid.f[1];
    b.ws = mid.f[2];
    b.u = vin[0];
    b.v = vin[1];
    b.w = vin[2];
    cudaError_t r;
    if ((r = plain_front(g, b, s)) != cudaSuccess) return r;
    if (e.conv) {
        if ((r = step_pressure(e, pafter, s)) != cudaSuccess) return r;
    } else {
        if ((r = plain_pressure(g, b, e.jacobi_iters, par, s)) != cudaSuccess) return r;
        *pafter = *par ? b.p1 : b.p0;
    }
    b.u = vout[0];
    b.v = vout[1];
    b.w = vout[2];
    if ((r = plain_correct(g, b, *pafter, s)) != cudaSuccess) return r;
    const int* dirs = sweep_order(istep);
    const float* velof[3] = {b.u, b.v, b.w};
    if ((r = fct_launch_to(g, dirs[0], false, Fin, mid.f[3], velof[dirs[0]], s)) != cudaSuccess ||
        (r = fct_launch_to(g, dirs[1], false, mid.f[3], mid.f[4], velof[dirs[1]], s)) != cudaSuccess)
        return r;
    // the step's final F: the next step's input (a reversed step reads only
    // F before each sweep); Fout == nullptr when no step follows
    if (Fout && (r = fct_launch_to(g, dirs[2], true, mid.f[4], Fout, velof[dirs[2]], s)) != cudaSuccess) return r;
    return cudaSuccess;
}

// One reversed step: the adjoint kernels on the step's data d.
cudaError_t reverse_step(AdjEngine& e, const StepData& d, int istep, cudaStream_t s) {
    const Geom& g = e.g;
    cudaError_t r;
    const int* dirs = sweep_order(istep);
    double* lvelof[3] = {e.lu, e.lv, e.lw};
    // F boundary copies
    {
        const dim3 b(16, 16);
        k_adj_bcF_z<<<dim3((g.nx + 2 + 15) / 16, (g.ny + 2 + 15) / 16), b, 0, s>>>(g, e.lF);
        k_adj_bcF_x<<<dim3((g.ny + 2 + 15) / 16, (g.nz + 2 + 15) / 16), b, 0, s>>>(g, e.lF);
        k_adj_bcF_y<<<dim3((g.nx + 2 + 15) / 16, (g.nz + 2 + 15) / 16), b, 0, s>>>(g, e.lF);
    }
    // the three sweeps, last first
    for (int q = 2; q >= 0; --q) {
        const int a = dirs[q];
        r = a == 0 ? sweep_adjoint<0>(e, d.Fsw[q], d.vel[0], lvelof[0], s)
                   : (a == 1 ? sweep_adjoint<1>(e, d.Fsw[q], d.vel[1], lvelof[1], s)
                             : sweep_adjoint<2>(e, d.Fsw[q], d.vel[2], lvelof[2], s));
        if (r != cudaSuccess) return r;
    }
    // velocity boundary copies, then the correction
    {
        const dim3 b(16, 16);
        k_adj_bcv_z<<<dim3((g.nx + 2 + 15) / 16, (g.ny + 2 + 15) / 16), b, 0, s>>>(g, e.lu, e.lv, e.lw);
        k_adj_bcv_x<<<dim3((g.ny + 2 + 15) / 16, (g.nz + 2 + 15) / 16), b, 0, s>>>(g, e.lu, e.lv, e.lw);
        k_adj_bcv_y<<<dim3((g.nx + 2 + 15) / 16, (g.nz + 2 + 15) / 16), b, 0, s>>>(g, e.lu, e.lv, e.lw);
    }
    const Range I = interior(g);
    const dim3 gi = grid_of(I);
    // plain step with sweeps: the update also applies the later step's
    // deferred last transposed stage and this step's first one (mu0 into the
    // other lp buffer, lrhs = mu0)
    const bool fuse = !e.conv && e.jacobi_iters > 0;
    if (fuse) {
        k_adj_update<true><<<gi, kBlk, 0, s>>>(g, I, d.F, d.p, e.lu, e.lv, e.lw, e.lp[e.lp_cur], e.lrho,
                                               e.lp_pending ? 1 : 0, e.inv_ap, e.lp[e.lp_cur ^ 1], e.lrhs);
        e.lp_cur ^= 1;
    } else {
        k_adj_update<false><<<gi, kBlk, 0, s>>>(g, I, d.F, d.p, e.lu, e.lv, e.lw, e.lp[e.lp_cur], e.lrho, 0,
                                                e.inv_ap, nullptr, nullptr);
    }
    // lu, lv, lw now hold the adjoints of u*, v*, w*; the start velocity's
    // adjoint accumulates in the cleared second set
    for (double* l : {e.lus, e.lvs, e.lws})
        if ((r = cudaMemsetAsync(l, 0, e.elems * sizeof(double), s)) != cudaSuccess) return r;
    // the pressure solve reversed: convergent modes -- lrhs = the mean-free
    // solution of A mu = lp - mean(lp) (warm start: the previous step's), and
    // the state pressure (only a warm start) gets no adjoint; plain -- the
    // Jacobi sweeps transposed (on mu = lambda / ap)
    if (e.conv) {
        r = mg_solve64(g, e.mg_adj, e.lp[e.lp_cur], e.lrhs, e.tol, e.max_outer, nullptr, s, e.cap);
        if (r != cudaSuccess) return r;
        if ((r = cudaMemsetAsync(e.lp[e.lp_cur], 0, e.elems * sizeof(double), s)) != cudaSuccess) return r;
    } else if (e.jacobi_iters > 0) {
        // stages 1 .. iters - 1 (mode 1), two per launch; stage 0 ran in the
        // update, the last one (mode 2) is deferred to the update of the
        // earlier step, or to the end of the reverse pass
        const int n1 = e.jacobi_iters - 1;
        // chunks of up to 24 planes, shorter on small grids (about 600 blocks)
        const long long cols = (long long)((g.nx + AJ_TX - 1) / AJ_TX) * ((g.ny + AJ_TY - 1) / AJ_TY);
        const int target = (int)(g.nz * cols / 600), len = target < 1 ? 1 : (target > 24 ? 24 : target);
        const int nch = (g.nz + len - 1) / len, kchunk = (g.nz + nch - 1) / nch;
        const dim3 gj((g.nx + AJ_TX - 1) / AJ_TX, (g.ny + AJ_TY - 1) / AJ_TY, (g.nz + kchunk - 1) / kchunk);
        const dim3 bj(AJ_TX, AJ_TY);
        for (int q = 0; q < n1; q += 2) {
            const double* in = e.lp[e.lp_cur];
            double* out = e.lp[e.lp_cur ^ 1];
            if (q + 1 < n1)
                k_adj_jacobi2<1, 1><<<gj, bj, 0, s>>>(g, e.inv_ap, in, out, e.lrhs, kchunk);
            else
                k_adj_jacobi<<<gi, kBlk, 0, s>>>(g, I, e.inv_ap, in, out, e.lrhs, 1);
            e.lp_cur ^= 1;
        }
        e.lp_pending = true;
    }
    // rhs, advection, rho and nu
    k_adj_advect<<<gi, kBlk, 0, s>>>(g, I, d.F, d.u, d.v, d.w, d.us, d.vs, d.ws, e.lrhs, e.conv || e.jacobi_iters > 0,
                                     e.lu, e.lv, e.lw, e.lus, e.lvs, e.lws, e.lrho, e.lF, e.d_partial);
    std::swap(e.lu, e.lus);
    std::swap(e.lv, e.lvs);
    std::swap(e.lw, e.lws);
    return cudaGetLastError();
}

}  // namespace

int adj_kernels_per_step(const AdjEngine& e) {
    // Per reversed step: the replay's forward step (front 2, pressure,
    // correction 1, three sweeps), the recomputation when the intermediates
    // are not kept (front 2, pressure, correction 1, two sweeps), and the
    // adjoint kernels: F copies 3, the three sweep adjoints (1 launch each when
    // fused, else 8), velocity copies 3, correction 1 (with the first and the
    // deferred last transposed Jacobi stage), the other iters - 1 stages two
    // per launch, rhs with advection 1.  The convergent modes' pressure solves
    // (multigrid graphs) are not counted.
    const Geom& g = e.g;
    const int P = e.conv ? 0 : plain_phase_launches(e.g, PHASE_JACOBI, e.jacobi_iters);
    int sweeps = 0;
    const int len[3] = {g.nx, g.ny, g.nz};
    const long lines[3] = {(long)g.ny * g.nz, (long)g.nx * g.nz, (long)g.nx * g.ny};
    for (int a = 0; a < 3; ++a)
        sweeps += (e.fct_march == 2 || (e.fct_march && lines[a] >= FM_MIN_LINES) ||
                   fa_smem_bytes(2, len[a]) <= fa_smem_limit())
                      ? 1
                      : 8;
    const int replay = 2 + P + 1 + 3;
    const int recompute = e.keep ? 0 : 2 + P + 1 + 2;
    const int jac = (!e.conv && e.jacobi_iters > 0) ? e.jacobi_iters / 2 : 0;
    return replay + recompute + 3 + sweeps + 3 + 1 + jac + 1;
}

cudaError_t adj_create(const Geom& g, int jacobi_iters, int mg_mode, double tol, int max_outer, AdjEngine* e,
                       cudaStream_t s) {
    *e = AdjEngine{};
    e->g = g;
    e->jacobi_iters = jacobi_iters;
    e->conv = mg_mode != 0;
    e->tol = tol;
    e->max_outer = max_outer;
    // sweep adjoint kernel: by grid size, or forced by VOF_ADJ_SWEEP=march|shared
    e->fct_march = 1;
    if (const char* v = getenv("VOF_ADJ_SWEEP")) {
        if (!strcmp(v, "march")) e->fct_march = 2;
        else if (!strcmp(v, "shared")) e->fct_march = 0;
    }
    e->elems = (size_t)g.plane * (g.nz + 2);
    cudaError_t r;
    auto alloc = [&](void** p, size_t nb) -> cudaError_t {
        cudaError_t q = cudaMalloc(p, nb);
        if (q != cudaSuccess) {
            *p = nullptr;
            return q;
        }
        e->bytes += nb;
        return cudaMemsetAsync(*p, 0, nb, s);
    };
    const size_t fb = e->elems * sizeof(float), db = e->elems * sizeof(double);
    float** f32[] = {&e->wb.F, &e->wb.u, &e->wb.v, &e->wb.w, &e->wb.us, &e->wb.vs, &e->wb.ws, &e->wb.rhs, &e->wb.p0,
                     &e->wb.p1, &e->wb.p2, &e->Fin1, &e->Fin2, &e->Ftd, &e->A, &e->C, &e->rp, &e->rm};
    for (float** p : f32)
        if ((r = alloc((void**)p, fb)) != cudaSuccess) return r;
    double** f64[] = {&e->lF, &e->lu, &e->lv, &e->lw, &e->lp[0], &e->lp[1], &e->lus, &e->lvs, &e->lws, &e->lrhs,
                      &e->lrho, &e->lnu, &e->lX, &e->lown, &e->lmx, &e->lmn, &e->lpp, &e->lpm, &e->ldv, &e->lterm,
                      &e->lLF, &e->lA};
    for (double** p : f64)
        if ((r = alloc((void**)p, db)) != cudaSuccess) return r;
    if ((r = alloc((void**)&e->sel, e->elems)) != cudaSuccess) return r;
    if ((r = alloc((void**)&e->status, sizeof(int))) != cudaSuccess) return r;
    const dim3 gi = grid_of(interior(g));
    e->npartial = (int)(gi.x * gi.y * gi.z);
    const Range full{0, g.nx + 1, 0, g.ny + 1, 0, g.nz + 1};
    const dim3 gf = grid_of(full);
    const int nseed = (int)(gf.x * gf.y * gf.z);
    const int np = 3 * e->npartial > nseed ? 3 * e->npartial : nseed;
    if ((r = alloc((void**)&e->d_partial, sizeof(double) * np)) != cudaSuccess) return r;
    if ((r = alloc((void**)&e->d_sums, sizeof(double) * 4)) != cudaSuccess) return r;
    if ((r = cudaMallocHost((void**)&e->h_sums, sizeof(double) * 4)) != cudaSuccess) {
        e->h_sums = nullptr;
        return r;
    }
    // 1 / ap for the 64 wall-flag combinations (the forward's FP32 ap, in its order)
    for (int f = 0; f < 64; ++f) {
        const float cx = g.dxi * g.dxi, cy = g.dyi * g.dyi, cz = g.dzi * g.dzi;
        const bool i1 = f & 1, inx = f & 2, j1 = f & 4, jny = f & 8, k1 = f & 16, knz = f & 32;
        const float ae = inx ? 0.0f : cx, aw = i1 ? 0.0f : cx, an = jny ? 0.0f : cy, as = j1 ? 0.0f : cy;
        const float af = knz ? 0.0f : cz, ab = k1 ? 0.0f : cz;
        const float ap = -(ae + aw + an + as + af + ab);
        e->inv_ap.v[f] = ap != 0.0f ? 1.0 / (double)ap : 0.0;
    }
    const float* mapped[4] = {e->wb.p0, e->wb.p1, e->wb.p2, e->wb.rhs};
    for (int q = 0; q < 4; ++q)
        if ((r = jacobi_tb_maps(g, mapped[q], &e->maps[q])) != cudaSuccess) return r;
    if (e->conv) {
        if ((r = alloc((void**)&e->p64, db)) != cudaSuccess) return r;
        if ((r = mg_create(g, mg_mode, &e->mg_fwd, s, &e->bytes)) != cudaSuccess) return r;
        if ((r = mg_create(g, mg_mode, &e->mg_adj, s, &e->bytes)) != cudaSuccess) return r;
        if ((r = cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking)) != cudaSuccess) {
            e->cap = nullptr;
            return r;
        }
    }
    e->wb.maps = e->maps;
    e->wb.status = e->status;
    return cudaStreamSynchronize(s);
}

static void free_states(AdjState* st, int n) {
    if (!st) return;
    for (int m = 0; m < n; ++m) {
        for (int q = 0; q < 5; ++q)
            if (st[m].f[q]) cudaFree(st[m].f[q]);
        if (st[m].p64) cudaFree(st[m].p64);
    }
    delete[] st;
}

static void free_mid(AdjMid* m, int n) {
    if (!m) return;
    for (int q = 0; q < n; ++q)
        for (int t = 0; t < 5; ++t)
            if (m[q].f[t]) cudaFree(m[q].f[t]);
    delete[] m;
}

// Free the tape (checkpoints, segment states, intermediates).
static void free_tape(AdjEngine* e) {
    free_states(e->cp, e->ncp);
    free_states(e->seg, e->every);
    free_mid(e->mid, e->every);
    for (int i = 0; i < e->nkept; ++i) {
        free_states(e->kseg[i], e->every);
        free_mid(e->kmid[i], e->every);
        e->kseg[i] = nullptr;
        e->kmid[i] = nullptr;
        e->kept[i] = false;
    }
    e->nkept = 0;
    e->cp = e->seg = nullptr;
    e->mid = nullptr;
    e->ncp = 0;
    e->keep = 0;
    e->tape_bytes = 0;
}

void adj_destroy(AdjEngine* e) {
    free_tape(e);
    float* f32[] = {e->wb.F, e->wb.u, e->wb.v, e->wb.w, e->wb.us, e->wb.vs, e->wb.ws, e->wb.rhs, e->wb.p0,
                    e->wb.p1, e->wb.p2, e->Fin1, e->Fin2, e->Ftd, e->A, e->C, e->rp, e->rm};
    for (float* p : f32)
        if (p) cudaFree(p);
    double* f64[] = {e->lF, e->lu, e->lv, e->lw, e->lp[0], e->lp[1], e->lus, e->lvs, e->lws, e->lrhs, e->lrho,
                     e->lnu, e->lX, e->lown, e->lmx, e->lmn, e->lpp, e->lpm, e->ldv, e->lterm, e->lLF, e->lA,
                     e->d_partial, e->d_sums};
    for (double* p : f64)
        if (p) cudaFree(p);
    if (e->sel) cudaFree(e->sel);
    if (e->status) cudaFree(e->status);
    if (e->p64) cudaFree(e->p64);
    if (e->conv) {
        mg_destroy(&e->mg_fwd);
        mg_destroy(&e->mg_adj);
    }
    if (e->cap) cudaStreamDestroy(e->cap);
    if (e->h_sums) cudaFreeHost(e->h_sums);
    *e = AdjEngine{};
}

// n states; entries below `first` stay unallocated (null).
static cudaError_t alloc_states(AdjState*& st, int n, int first, size_t elems, bool with_p64, size_t* bytes) {
    st = new (std::nothrow) AdjState[n];
    if (!st) return cudaErrorMemoryAllocation;
    for (int m = 0; m < n; ++m) {
        for (int q = 0; q < 5; ++q) st[m].f[q] = nullptr;
        st[m].p64 = nullptr;
    }
    for (int m = first; m < n; ++m) {
        for (int q = 0; q < 5; ++q) {
            cudaError_t r = cudaMalloc((void**)&st[m].f[q], elems * sizeof(float));
            if (r != cudaSuccess) {
                st[m].f[q] = nullptr;
                return r;
            }
            *bytes += elems * sizeof(float);
        }
        if (with_p64) {
            cudaError_t r = cudaMalloc((void**)&st[m].p64, elems * sizeof(double));
            if (r != cudaSuccess) {
                st[m].p64 = nullptr;
                return r;
            }
            *bytes += elems * sizeof(double);
        }
    }
    return cudaSuccess;
}

static cudaError_t alloc_mid(AdjMid*& m, int n, size_t elems, size_t* bytes, cudaStream_t s) {
    m = new (std::nothrow) AdjMid[n];
    if (!m) return cudaErrorMemoryAllocation;
    for (int q = 0; q < n; ++q)
        for (int t = 0; t < 5; ++t) m[q].f[t] = nullptr;
    for (int q = 0; q < n; ++q)
        for (int t = 0; t < 5; ++t) {
            cudaError_t r = cudaMalloc((void**)&m[q].f[t], elems * sizeof(float));
            if (r != cudaSuccess) {
                m[q].f[t] = nullptr;
                return r;
            }
            *bytes += elems * sizeof(float);
            if ((r = cudaMemsetAsync(m[q].f[t], 0, elems * sizeof(float), s)) != cudaSuccess) return r;
        }
    return cudaSuccess;
}

cudaError_t adj_tape(AdjEngine* e, int istep0, int nsteps, int every, cudaStream_t s) {
    if (every <= 0) {
        every = 1;
        while ((long long)every * every < nsteps) ++every;
    }
    if (every > nsteps) every = nsteps > 0 ? nsteps : 1;
    const int ncp = nsteps > 0 ? (nsteps + every - 1) / every : 0;
    const size_t fb = e->elems * sizeof(float), db = e->elems * sizeof(double);
    // keep the intermediates?  (checkpoints + segment states 1.. + intermediates)
    bool keep = false;
    if (e->policy == ADJ_STORE_KEEP) {
        keep = true;
    } else if (e->policy == ADJ_STORE_AUTO) {
        size_t fr = 0, tot = 0;
        const size_t need = (size_t)ncp * (5 * fb + (e->conv ? db : 0)) + (size_t)(every - 1) * 5 * fb +
                            (size_t)every * 5 * fb;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
            // (the current tape's memory comes back when it is reallocated)
            keep = need + tot / 32 <= fr + e->tape_bytes;
        }
    }
    if (e->cp && (ncp != e->ncp || every != e->every || (int)keep != e->keep)) free_tape(e);
    cudaError_t r;
    if (!e->cp && ncp > 0) {
        e->ncp = ncp;
        e->every = every;
        e->keep = keep;
        if ((r = alloc_states(e->cp, ncp, 0, e->elems, e->conv, &e->tape_bytes)) != cudaSuccess) return r;
        // kept tapes: a segment's first state is its checkpoint, and the
        // replay carries the FP64 warm start itself
        if ((r = alloc_states(e->seg, every, keep ? 1 : 0, e->elems, e->conv && !keep, &e->tape_bytes)) !=
            cudaSuccess)
            return r;
        if (keep && (r = alloc_mid(e->mid, every, e->elems, &e->tape_bytes, s)) != cudaSuccess) return r;
    }
    // further kept segments, where the record can keep them and memory
    // allows (a tape that keeps intermediates, FP32 Jacobi with an even sweep
    // count): one set per segment before the last, from the last backwards
    const bool want = keep && !e->conv && e->jacobi_iters % 2 == 0 && ncp >= 2;
    int nwant = want ? ncp - 1 : 0;
    if (nwant > AdjEngine::MAX_KEPT) nwant = AdjEngine::MAX_KEPT;
    while (e->nkept > nwant) {
        const int i = --e->nkept;
        free_states(e->kseg[i], e->every);
        free_mid(e->kmid[i], e->every);
        e->kseg[i] = nullptr;
        e->kmid[i] = nullptr;
    }
    while (e->nkept < nwant) {
        size_t fr = 0, tot = 0;
        const size_t need = (size_t)(2 * every - 1) * 5 * fb;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess || need + tot / 32 > fr) break;
        const int i = e->nkept;
        size_t bk = 0;
        r = alloc_states(e->kseg[i], every, 1, e->elems, false, &bk);
        if (r == cudaSuccess) r = alloc_mid(e->kmid[i], every, e->elems, &bk, s);
        if (r != cudaSuccess) {  // (only an optimisation: go without it)
            free_states(e->kseg[i], every);
            free_mid(e->kmid[i], every);
            e->kseg[i] = nullptr;
            e->kmid[i] = nullptr;
            cudaGetLastError();
            break;
        }
        e->tape_bytes += bk;
        ++e->nkept;
    }
    e->istep0 = istep0;
    e->nsteps = nsteps;
    e->every = every;
    e->recorded = false;
    e->tail_kept = false;
    e->tail_p = nullptr;
    for (int i = 0; i < AdjEngine::MAX_KEPT; ++i) e->kept[i] = false;
    return cudaSuccess;
}

int adj_segment_first(const AdjEngine& e, int m) {
    if (m >= e.ncp) return e.nsteps;
    const long long f = (long long)e.nsteps - (long long)(e.ncp - m) * e.every;
    return f > 0 ? (int)f : 0;
}

bool adj_can_record_tail(const AdjEngine& e) { return e.keep && !e.conv && e.jacobi_iters % 2 == 0 && e.ncp > 0; }

// One step of a kept segment replay: step q of the segment that starts at
// `first` (count steps), from the engine's buffers (q == 0: loaded from the
// checkpoint) or segment state seg[q], into seg[q + 1] or the engine's
// buffers (last step), keeping its intermediates in mid[q]; the pressure after
// the sweeps is copied into seg[q + 1].  *pa: where that pressure is
// afterwards.
static cudaError_t replay_kept(AdjEngine& e, AdjState* seg, AdjMid* mid, int first, int count, int q, int* par,
                               const float** pa, cudaStream_t s, bool final_F = true) {
    float* const* vs = q == 0 ? nullptr : seg[q].f + 1;
    float* const vin[3] = {q == 0 ? e.wb.u : vs[0], q == 0 ? e.wb.v : vs[1], q == 0 ? e.wb.w : vs[2]};
    float* const* vn = q + 1 < count ? seg[q + 1].f + 1 : nullptr;
    float* const vout[3] = {vn ? vn[0] : e.wb.u, vn ? vn[1] : e.wb.v, vn ? vn[2] : e.wb.w};
    const float* Fin = q == 0 ? e.wb.F : seg[q].f[0];
    float* Fout = q + 1 < count ? seg[q + 1].f[0] : (final_F ? e.wb.F : nullptr);
    cudaError_t r = replay_step_keep(e, e.istep0 + first + q, mid[q], Fin, Fout, vin, vout, par, pa, s);
    if (r == cudaSuccess && q + 1 < count) {
        r = copy_field(seg[q + 1].f[4], *pa, e.elems, s);
        *pa = seg[q + 1].f[4];
    }
    return r;
}

cudaError_t adj_record_tail(AdjEngine* e, const AdjState& out, float* const extra[4], cudaStream_t s) {
    if (!adj_can_record_tail(*e)) return cudaErrorNotSupported;
    const int m = e->ncp - 1;
    const int first = adj_segment_first(*e, m), count = e->nsteps - first;
    cudaError_t r = load_state(*e, e->cp[m], s);
    int par = 0;
    const float* pa = nullptr;
    for (int q = 0; q < count && r == cudaSuccess; ++q)
        r = replay_kept(*e, e->seg, e->mid, first, count, q, &par, &pa, s);
    if (r != cudaSuccess) return r;
    const float* src[5] = {e->wb.F, e->wb.u, e->wb.v, e->wb.w, pa};
    for (int q = 0; q < 5; ++q)
        if ((r = copy_field(out.f[q], src[q], e->elems, s)) != cudaSuccess) return r;
    const float* xs[4] = {e->mid[count - 1].f[0], e->mid[count - 1].f[1], e->mid[count - 1].f[2], e->wb.rhs};
    for (int q = 0; q < 4; ++q)
        if (extra[q] && (r = copy_field(extra[q], xs[q], e->elems, s)) != cudaSuccess) return r;
    e->tail_kept = true;
    e->tail_p = pa;
    return cudaSuccess;
}

bool adj_can_keep(const AdjEngine& e, int m) {
    const int i = e.ncp - 2 - m;
    return adj_can_record_tail(e) && i >= 0 && i < e.nkept && e.kseg[i] && e.kmid[i];
}

cudaError_t adj_record_keep(AdjEngine* e, int m, const AdjState& out, cudaStream_t s) {
    if (!adj_can_keep(*e, m)) return cudaErrorNotSupported;
    const int i = e->ncp - 2 - m;
    const int first = adj_segment_first(*e, m), count = adj_segment_first(*e, m + 1) - first;
    cudaError_t r = load_state(*e, e->cp[m], s);
    int par = 0;
    const float* pa = nullptr;
    for (int q = 0; q < count && r == cudaSuccess; ++q)
        r = replay_kept(*e, e->kseg[i], e->kmid[i], first, count, q, &par, &pa, s);
    if (r != cudaSuccess) return r;
    const float* src[5] = {e->wb.F, e->wb.u, e->wb.v, e->wb.w, pa};
    for (int q = 0; q < 5; ++q)
        if ((r = copy_field(out.f[q], src[q], e->elems, s)) != cudaSuccess) return r;
    e->kept[i] = true;
    return cudaSuccess;
}

cudaError_t adj_save(AdjEngine* e, int m, const AdjState& x, cudaStream_t s) {
    if (m < 0 || m >= e->ncp) return cudaErrorInvalidValue;
    cudaError_t r;
    for (int q = 0; q < 5; ++q)
        if ((r = copy_field(e->cp[m].f[q], x.f[q], e->elems, s)) != cudaSuccess) return r;
    if (e->conv)
        return cudaMemcpyAsync(e->cp[m].p64, x.p64, e->elems * sizeof(double), cudaMemcpyDeviceToDevice, s);
    return cudaSuccess;
}

cudaError_t adj_backward(AdjEngine* e, const AdjState& fin, const double box[6], double* loss, double grad_g[3],
                         cudaStream_t s) {
    const Geom& g = e->g;
    cudaError_t r;
    // seed and loss
    double* zero[] = {e->lu, e->lv, e->lw, e->lp[0], e->lp[1], e->lrho, e->lrhs};
    for (double* p : zero)
        if ((r = cudaMemsetAsync(p, 0, e->elems * sizeof(double), s)) != cudaSuccess) return r;
    if ((r = cudaMemsetAsync(e->d_sums, 0, 4 * sizeof(double), s)) != cudaSuccess) return r;
    e->lp_cur = 0;
    e->lp_pending = false;
    {
        const Range full{0, g.nx + 1, 0, g.ny + 1, 0, g.nz + 1};
        const dim3 gf = grid_of(full);
        Box6 b;
        for (int q = 0; q < 6; ++q) b.b[q] = box[q];
        k_seed<<<gf, kBlk, 0, s>>>(g, full, b, fin.f[0], e->lF, e->d_partial);
        k_fold_add<<<1, 256, 0, s>>>(e->d_partial, (int)(gf.x * gf.y * gf.z), 1, e->d_sums + 3);
        if ((r = cudaGetLastError()) != cudaSuccess) return r;
        if ((r = cudaMemsetAsync(e->d_partial, 0, sizeof(double) * 3 * e->npartial, s)) != cudaSuccess) return r;
    }
    // segments, last first
    for (int m = e->ncp - 1; m >= 0; --m) {
        const int first = adj_segment_first(*e, m);
        const int count = adj_segment_first(*e, m + 1) - first;
        if (e->keep) {
            // replay every step of the segment from checkpoint m, keeping its
            // intermediates and the states after steps 0 .. count - 2; the
            // record did so already for the last segment when tail_kept, and
            // for the ones before it that have a kept set
            const bool tail = m == e->ncp - 1 && e->tail_kept;
            const int ki = e->ncp - 2 - m;
            const bool k2 = ki >= 0 && ki < e->nkept && e->kept[ki];
            AdjState* const seg = k2 ? e->kseg[ki] : e->seg;
            AdjMid* const mid = k2 ? e->kmid[ki] : e->mid;
            // the state after the segment's last step: the replay's buffers,
            // or checkpoint m + 1 for a kept set
            const AdjState wbs{{e->wb.F, e->wb.u, e->wb.v, e->wb.w, nullptr}, nullptr};
            const AdjState& after = k2 ? e->cp[m + 1] : wbs;
            if (!tail && !k2 && (r = load_state(*e, e->cp[m], s)) != cudaSuccess) return r;
            int par = 0;
            const float* pafter[64];
            const float** pa = count <= 64 ? pafter : new (std::nothrow) const float*[count];
            if (!pa) return cudaErrorMemoryAllocation;
            if (tail || k2) {
                for (int q = 0; q < count; ++q)
                    pa[q] = q + 1 < count ? seg[q + 1].f[4] : (k2 ? after.f[4] : e->tail_p);
                if (tail) e->tail_kept = false;  // the engine's buffers are reused from here on
            } else {
                for (int q = 0; q < count && r == cudaSuccess; ++q)  // (the segment's final F is not needed)
                    r = replay_kept(*e, seg, mid, first, count, q, &par, &pa[q], s, false);
            }
            // reverse: step q's next state is seg[q + 1], or `after` for the
            // segment's last step
            for (int q = count - 1; q >= 0 && r == cudaSuccess; --q) {
                const AdjState& x = q == 0 ? e->cp[m] : seg[q];
                const AdjMid& md = mid[q];
                const float* nu = q + 1 < count ? seg[q + 1].f[1] : after.f[1];
                const float* nv = q + 1 < count ? seg[q + 1].f[2] : after.f[2];
                const float* nw = q + 1 < count ? seg[q + 1].f[3] : after.f[3];
                const StepData d{x.f[0], x.f[1], x.f[2], x.f[3], md.f[0], md.f[1], md.f[2], pa[q],
                                 {nu, nv, nw}, {x.f[0], md.f[3], md.f[4]}};
                r = reverse_step(*e, d, e->istep0 + first + q, s);
            }
            if (pa != pafter) delete[] pa;
            if (r != cudaSuccess) return r;
            continue;
        }
        // the segment's states: checkpoint m, then count - 1 steps with the engine's buffers
        for (int q = 0; q < 5; ++q)
            if ((r = copy_field(e->seg[0].f[q], e->cp[m].f[q], e->elems, s)) != cudaSuccess) return r;
        if (e->conv && (r = cudaMemcpyAsync(e->seg[0].p64, e->cp[m].p64, e->elems * sizeof(double),
                                            cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
            return r;
        if (count > 1) {
            if ((r = load_state(*e, e->seg[0], s)) != cudaSuccess) return r;
            int par = 0;
            for (int q = 1; q < count; ++q) {
                const int istep = e->istep0 + first + q - 1;
                if (e->conv) {
                    const float* pa = nullptr;
                    if ((r = plain_front(g, e->wb, s)) != cudaSuccess || (r = step_pressure(*e, &pa, s)) != cudaSuccess ||
                        (r = plain_back(g, e->wb, istep, pa, s)) != cudaSuccess)
                        return r;
                } else if ((r = plain_step(g, e->wb, istep, e->jacobi_iters, &par, s)) != cudaSuccess) {
                    return r;
                }
                const float* src[5] = {e->wb.F, e->wb.u, e->wb.v, e->wb.w, par ? e->wb.p1 : e->wb.p0};
                for (int t = 0; t < 5; ++t)
                    if ((r = copy_field(e->seg[q].f[t], src[t], e->elems, s)) != cudaSuccess) return r;
                if (e->conv && (r = cudaMemcpyAsync(e->seg[q].p64, e->p64, e->elems * sizeof(double),
                                                    cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
                    return r;
            }
        }
        for (int q = count - 1; q >= 0; --q) {
            StepData d;
            if ((r = recompute_step(*e, e->seg[q], e->istep0 + first + q, &d, s)) != cudaSuccess ||
                (r = reverse_step(*e, d, e->istep0 + first + q, s)) != cudaSuccess)
                return r;
        }
    }
    if (e->lp_pending) {  // the first step's deferred last Jacobi stage: the initial pressure's adjoint
        const Range I = interior(g);
        k_adj_jacobi<<<grid_of(I), kBlk, 0, s>>>(g, I, e->inv_ap, e->lp[e->lp_cur], e->lp[e->lp_cur ^ 1], e->lrhs, 2);
        e->lp_cur ^= 1;
        e->lp_pending = false;
    }
    k_fold_add<<<1, 256, 0, s>>>(e->d_partial, e->npartial, 3, e->d_sums);
    if ((r = cudaGetLastError()) != cudaSuccess) return r;
    if ((r = cudaMemcpyAsync(e->h_sums, e->d_sums, 4 * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return r;
    if ((r = cudaStreamSynchronize(s)) != cudaSuccess) return r;
    if (grad_g)
        for (int q = 0; q < 3; ++q) grad_g[q] = e->h_sums[q];
    if (loss) *loss = e->h_sums[3];
    return cudaSuccess;
}

}  // namespace vof
