// fct_line.cuh -- per-cell expressions of one FCT sweep along a grid line
// (fct_{x,y,z}_sweep_stage1..4, voftrial1.cu:509-905), shared by the forward
// sweep kernel (fct_sweep.cu) and the sweep adjoint (adjoint.cu), which
// recomputes the forward's stage values.  Both translation units are compiled
// with -fmad=false, so these expressions give the same bits in both.
//
// Length factors of the reference, per sweep (x | y | z):
//   stage 1 flux term  (f_l - f_r)*dy*dz/vol | (f_l - f_r)*dy/(dx*dy) | (f_l - f_r)*dy*dx/vol
//   dv factor          dt*dy*dz              | dt*dx*dz               | dt*dx*dy
//   limiter q          *dx                   | *dx                    | *dz
//   stage 4 divisor    /dy                   | /dy                    | /dz
#pragma once
#include <cuda_runtime.h>

#include "vof_device.cuh"

namespace vof {
namespace fct {

// Per-sweep constants (the table above) and the IEEE reciprocals of the
// constant divisors, for div_rn_pre.
template <int AXIS>
struct Sweep {
    float dt, vol, dvfac, hq, h4, t1a, t1b, dxdy;
    float rvol, rh4, rdxdy;
    int n;

    __device__ Sweep(const Geom& g) {
        dt = g.dt;
        vol = g.dx * g.dy * g.dz;
        n = AXIS == 0 ? g.nx : (AXIS == 1 ? g.ny : g.nz);
        dvfac = AXIS == 0 ? g.dt * g.dy * g.dz : (AXIS == 1 ? g.dt * g.dx * g.dz : g.dt * g.dx * g.dy);
        hq = AXIS == 2 ? g.dz : g.dx;
        h4 = AXIS == 2 ? g.dz : g.dy;
        t1a = g.dy;                                    // first factor of the stage-1 flux term
        t1b = AXIS == 0 ? g.dz : (AXIS == 1 ? 0.0f : g.dx);
        dxdy = g.dx * g.dy;
        rvol = __frcp_rn(vol);
        rh4 = __frcp_rn(h4);
        rdxdy = __frcp_rn(dxdy);
    }

    // Stage-1 flux term from the low-order fluxes through the lower (fi) and
    // upper (fo) faces of a cell.
    __device__ __forceinline__ float term(float fi, float fo) const {
        if (AXIS == 1) return div_rn_pre((fi - fo) * t1a, dxdy, rdxdy);
        return div_rn_pre((fi - fo) * t1a * t1b, vol, rvol);
    }

    // Cell volume change from the velocities of its lower and upper faces.
    __device__ __forceinline__ float dv(float v_lo, float v_hi) const { return vol - dvfac * (v_hi - v_lo); }
};

// Low-order flux and antidiffusive flux through a face with velocity uf
// between cells with values FL (lower) and FR (upper), as fl_L / fl_H of the
// reference's stages 1-2.
__device__ __forceinline__ void flux(float uf, float FL, float FR, float dt, float& lo, float& a) {
    const float lo_ = (uf >= 0.0f) ? uf * dt * FL : uf * dt * FR;
    const float hi_ = (uf <= 0.0f) ? uf * dt * FL : uf * dt * FR;
    lo = lo_;
    a = hi_ - lo_;
}

// Stage 1: low-order update of a cell from its face fluxes; rdv = RN(1/dv).
// *inside: the unclamped value lies in [0, 1] (the clamp passes it through).
template <int AXIS>
__device__ __forceinline__ float ftd_from(const Sweep<AXIS>& S, float Fc, float lo_in, float lo_out, float dv,
                                         float rdv, bool* inside = nullptr) {
    float out = div_rn_pre((Fc + S.term(lo_in, lo_out)) * S.vol, dv, rdv);
    const bool clip = out > 1.0f || out < 0.0f;
    if (inside) *inside = !clip;
    if (clip) out = clamp01f(out);
    return out;
}

// Stage 2: Zalesak ratios of a cell from the Ftd of the cell and its two
// neighbours (tm, tc, tp) and the antidiffusive fluxes of its lower (al) and
// upper (ar) faces.
template <int AXIS>
__device__ __forceinline__ void limiter(const Sweep<AXIS>& S, float tm, float tc, float tp, float al,
                                        float ar, float& rp, float& rm) {
    const float fmx = fmaxf(tc, fmaxf(tm, tp));
    const float fmn = fminf(tc, fminf(tm, tp));
    // rp = pp > 0 ? fminf(1, qp/pp) : 0, skipping the division when
    // qp >= pp (then qp/pp >= 1 and its rounding is >= 1 too).
    const float pp = fmaxf(0.0f, al) - fminf(0.0f, ar);
    const float qp = (fmx - tc) * S.hq;
    rp = 0.0f;
    if (pp > 0.0f) rp = (qp >= pp) ? 1.0f : fminf(1.0f, qp / pp);
    const float pm = fmaxf(0.0f, ar) - fminf(0.0f, al);
    const float qm = (tc - fmn) * S.hq;
    rm = 0.0f;
    if (pm > 0.0f) rm = (qm >= pm) ? 1.0f : fminf(1.0f, qm / pm);
}

// Stage 3: limiter of a face from the ratios of its lower and upper cells.
__device__ __forceinline__ float face_limit(float af, float rp_lo, float rm_lo, float rp_hi, float rm_hi) {
    return (af >= 0.0f) ? fminf(rp_hi, rm_lo) : fminf(rp_lo, rm_hi);
}

// Stage 4 before the final clamp: Ftd - ((a_hi c_hi - a_lo c_lo) / h4) vol / dv.
template <int AXIS>
__device__ __forceinline__ float stage4(const Sweep<AXIS>& S, float ftd, float a_lo, float c_lo, float a_hi,
                                        float c_hi, float dv, float rdv) {
    return ftd - div_rn_pre(div_rn_pre(a_hi * c_hi - a_lo * c_lo, S.h4, S.rh4) * S.vol, dv, rdv);
}

}  // namespace fct
}  // namespace vof
