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
// quotients.  Method: P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990 -- with
// rd = RN(1/d) and q0 = RN(x*rd) (within one ulp of x/d), the remainder
// r = x - q0*d is exact in one FMA and q1 = RN(q0 + r*rd) equals RN(x/d),
// provided nothing underflows or overflows.  Outside the range where that
// holds (tiny, huge or non-finite operands) the IEEE division is used, and
// +-0 numerators return x*rd, which carries the IEEE sign of 0/d.
// The IEEE division outside that range, kept out of line: it is rare, and
// inlined at every call site it would cost issue slots on every cell.
static __device__ __noinline__ float div_rn_slow(float x, float d) { return __fdiv_rn(x, d); }

__device__ __forceinline__ float div_rn_pre(float x, float d, float rd) {
    const float q0 = __fmul_rn(x, rd);
    const float r = __fmaf_rn(-q0, d, x);
    const float q1 = __fmaf_rn(r, rd, q0);
    const float ax = fabsf(x), aq = fabsf(q0);
    if (ax >= 0x1p-96f && aq >= 0x1p-96f && aq <= 0x1p+96f) return q1;
    if (x == 0.0f) return q0;
    return div_rn_slow(x, d);
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
