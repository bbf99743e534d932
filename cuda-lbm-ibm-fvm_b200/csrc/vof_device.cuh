// vof_device.cuh -- device-side geometry, padded layout and the scalar
// helpers of the reference (voftrial1.cu:52-70), shared by every kernel TU.
//
// Layout in HBM (internal, padded): cell (i,j,k), i in [0,nx+1] ... is at
//     ((k * py) + j) * px + i,   px = round_up(nx+2, 32), py = ny+2,
// so every x-row starts on a 128-byte boundary (TMA-legal strides, aligned
// vector loads).  The reference layout (voftrial1.cu:66-70) has px = nx+2 and
// is converted only at the C-ABI boundary (vof_upload / vof_download).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace vof {

// Everything a step kernel needs, passed by value (kernel parameter space).
struct Geom {
    int nx, ny, nz;      // interior cells
    int px, py;          // x pitch (elements) and y extent (ny+2) of the padded layout
    int plane;           // px*py
    // Physics/geometry constants, the float values of Params (voftrial1.cu:27-41).
    float dt, dx, dy, dz, dxi, dyi, dzi;
    float rho_l, rho_g, nu_l, nu_g;
    float gx, gy, gz;
    // 0.5*(rho_a + rho_b) for the pure-phase pairs (gas-gas, liquid-liquid,
    // gas-liquid) and dt divided by each, formed on the device at set-up.
    float rpair[3], qpair[3];
    // continuum surface force (extension, off unless csf): sigma from Params
    int csf;
    float sigma;
};

// #pragma unroll with a macro or template argument as the count.
#define VOF_PRAGMA_(x) _Pragma(#x)
#define VOF_UNROLL_(n) VOF_PRAGMA_(unroll n)
#define VOF_UNROLL(n) VOF_UNROLL_(n)

__host__ __device__ __forceinline__ int gidx(const Geom& g, int i, int j, int k) {
    return (k * g.py + j) * g.px + i;
}

__host__ __device__ __forceinline__ int clampi(int v, int lo, int hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

// median3f / clamp01f (voftrial1.cu:52-60).  The expression a+b+c-mx-mn is
// evaluated left to right in FP32, which rounds v to a multiple of 2^-23 on
// [0,1) and maps tiny negatives to tiny values of either sign; the step's
// results depend on that, so the expression is kept as it is.
__host__ __device__ __forceinline__ float median3f(float a, float b, float c) {
    const float mx = fmaxf(fmaxf(a, b), c);
    const float mn = fminf(fminf(a, b), c);
    return a + b + c - mx - mn;
}

__host__ __device__ __forceinline__ float clamp01f(float v) {
    return median3f(0.0f, 1.0f, v);
}

// Correctly rounded x / d from a precomputed rd = RN(1/d) (IEEE reciprocal,
// __frcp_rn), for divisors that are constant or reused across several
// quotients and whose reciprocal is a normal number (|d| < 2^126).
// Method: P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990 -- with rd = RN(1/d)
// and q0 = RN(x*rd) (within one ulp of x/d), the remainder r = x - q0*d is
// exact in one FMA and q1 = RN(q0 + r*rd) equals RN(x/d), provided nothing
// underflows or overflows.  The remainder is exact when x's exponent is at
// least e_min + p - 1 = -103 (S. Boldo, M. Daumas, "Representable correcting
// terms for possibly underflowing floating point operations", ARITH-16,
// 2003); the fast path asks |x| >= 2^-100 and a normal quotient,
// 2^-125 <= |q0| <= 2^96.
// Tiny numerators (|x| < 2^-100, as in the cells a pressure front has not
// reached yet) take div_rn_tiny below; +-0 numerators return x*rd, which
// carries the IEEE sign of 0/d; what is left (huge quotients, non-finite
// operands) takes the IEEE division, out of line: it is rare, and inlined at
// every call site it would cost issue slots on every cell.
static __device__ __noinline__ float div_rn_slow(float x, float d) { return __fdiv_rn(x, d); }

// RN(x/d) for 0 < |x| < 2^-36: the quotient of xs = x * 2^64 (exact) by
// Markstein's method, qs = RN(xs/d), scaled back by 2^-64.  When x/d is a
// normal number the scaling is exact and commutes with rounding.  When it is
// subnormal, y = RN(qs * 2^-64) rounds a second time, to the grid of 2^-149;
// rounding qs first can only change the result when qs * 2^-64 is exactly a
// midpoint of that grid (rounding is monotone and the midpoints lie on qs's
// finer grid).  That case is detected exactly -- qs - y*2^64 (exact: both are
// multiples of qs's quantum and they differ by at most 2^-86) equals +-2^-86
// -- and settled by the sign of the exact remainder xs - qs*d: zero means
// x/d is the midpoint itself (ties to even, as y already is), otherwise the
// result is the grid point on the remainder's side, (qs +- 2^-86) * 2^-64,
// exact.  Anything outside the scaled Markstein range goes to the IEEE
// division.  Tested bit for bit against __fdiv_rn over every exponent and on
// constructed subnormal midpoints.
__device__ __forceinline__ float div_rn_tiny(float x, float d, float rd) {
    if (!(fabsf(x) < 0x1p-36f)) return div_rn_slow(x, d);
    const float xs = __fmul_rn(x, 0x1p+64f);
    const float s0 = __fmul_rn(xs, rd);
    const float as = fabsf(s0);
    if (!(as >= 0x1p-125f && as <= 0x1p+96f)) return div_rn_slow(x, d);
    const float qs = __fmaf_rn(__fmaf_rn(-s0, d, xs), rd, s0);
    float y = __fmul_rn(qs, 0x1p-64f);
    const float d2 = __fsub_rn(qs, __fmul_rn(y, 0x1p+64f));
    if (fabsf(d2) == 0x1p-86f) {
        const float rem = __fmaf_rn(-qs, d, xs);
        if (rem != 0.0f) {
            const bool up = (rem > 0.0f) == (d > 0.0f);
            y = __fmul_rn(__fadd_rn(qs, up ? 0x1p-86f : -0x1p-86f), 0x1p-64f);
        }
    }
    return y;
}

__device__ __forceinline__ float div_rn_pre(float x, float d, float rd) {
    const float q0 = __fmul_rn(x, rd);
    const float r = __fmaf_rn(-q0, d, x);
    const float q1 = __fmaf_rn(r, rd, q0);
    const float ax = fabsf(x), aq = fabsf(q0);
    if (ax >= 0x1p-100f && aq >= 0x1p-125f && aq <= 0x1p+96f) return q1;
    if (x == 0.0f) return q0;
    return div_rn_tiny(x, d, rd);
}

// 1/x for a positive normal FP64 x, to within about one ulp (not always
// correctly rounded), for the FP64 partial derivatives of the adjoint; the
// FP32 forward never uses it.  Method: Newton-Raphson iteration for the
// reciprocal, r <- r + r (1 - x r), each step squaring the relative error,
// started from the PTX approximation rcp.approx.ftz.f64; two steps take the
// error of that approximation below the FP64 rounding error.
__device__ __forceinline__ double rcp64(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = __fma_rn(-x, r, 1.0);
    r = __fma_rn(r, e, r);
    e = __fma_rn(-x, r, 1.0);
    return __fma_rn(r, e, r);
}

// rho and nu from the volume fraction (voftrial1.cu:95-104), same operand order.
__device__ __forceinline__ float rho_of(const Geom& g, float F) {
    const float f = clamp01f(F);
    return g.rho_g * (1.0f - f) + g.rho_l * f;
}
__device__ __forceinline__ float nu_of(const Geom& g, float F) {
    const float f = clamp01f(F);
    return g.nu_l * f + g.nu_g * (1.0f - f);
}

}  // namespace vof
