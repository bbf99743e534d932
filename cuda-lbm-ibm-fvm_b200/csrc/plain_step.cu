// plain_step.cu -- the FP32 drop-in step (voftrial1.cu:1364-1401) as fused
// sm_100a kernels over the padded layout of vof_device.cuh.
//
// Arithmetic contract: every per-point expression keeps the reference's
// operand order, and this translation unit is compiled with -fmad=false, so
// no multiply-add is contracted into an FMA.  The results are therefore
// bit-identical to the reference's kernels compiled with -fmad=false and to
// the FP32 CPU restatement in oracle/ (built with -ffp-contract=off); the
// reference built with nvcc's default -fmad=true differs from both in the
// last bits of contracted expressions.
//
// Kernel map (reference kernels each one replaces):
//   k_predict      advect_{u,v,w}_kernel + cal_nu_rho_kernel   voftrial1.cu:95-104, 230-399
//   k_rhs          the rhs expression of solve_p_jacobi_kernel voftrial1.cu:418-422
//   k_jacobi       solve_p_jacobi_kernel (one sweep)           voftrial1.cu:401-439
//   k_correct      update_{u,v,w}_kernel + apply_bc_velocity   voftrial1.cu:441-493, 959-1051, 1107-1120
//   k_fct<AXIS,FINAL>  fct_{x,y,z}_sweep_stage1..4 (+ on the last sweep
//                  post_process_f_kernel and apply_bc_F)       voftrial1.cu:502-905, 1053-1105, 1122-1174
#include "plain_step.h"

#include <cuda_runtime.h>

namespace vof {

#ifndef VOF_PLAIN_NO_FMAD_CHECK
// Compile-time guard: the build must pass -fmad=false for this file.
#if defined(__CUDA_ARCH__) && !defined(VOF_FMAD_FALSE)
#error "plain_step.cu must be compiled with -fmad=false -DVOF_FMAD_FALSE"
#endif
#endif

// ---------------------------------------------------------------------------
// Momentum predictor: u*, v*, w* on the interior faces the reference updates
// (u: i in [imin+1, imax], j,k interior; v, w likewise), nu from F on the fly.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_predict(Geom g,
                                                 const float* __restrict__ F,
                                                 const float* __restrict__ u,
                                                 const float* __restrict__ v,
                                                 const float* __restrict__ w,
                                                 float* __restrict__ us,
                                                 float* __restrict__ vs,
                                                 float* __restrict__ ws) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;

    const int sy = g.px, sz = g.plane;
    const int id = gidx(g, i, j, k);
    const float nu = nu_of(g, __ldg(F + id));

    if (i >= 2) {  // advect_u_kernel, voftrial1.cu:230-285
        const float v_here = 0.25f * (__ldg(v + id - 1) + __ldg(v + id - 1 + sy) +
                                      __ldg(v + id) + __ldg(v + id + sy));
        const float w_here = 0.25f * (__ldg(w + id - 1) + __ldg(w + id - 1 + sz) +
                                      __ldg(w + id) + __ldg(w + id + sz));
        const float uc = __ldg(u + id);
        const float uim = __ldg(u + id - 1), uip = __ldg(u + id + 1);
        const float ujm = __ldg(u + id - sy), ujp = __ldg(u + id + sy);
        const float ukm = __ldg(u + id - sz), ukp = __ldg(u + id + sz);
        const float dudx = (uc > 0.0f) ? (uc - uim) * g.dxi : (uip - uc) * g.dxi;
        const float dudy = (v_here > 0.0f) ? (uc - ujm) * g.dyi : (ujp - uc) * g.dyi;
        const float dudz = (w_here > 0.0f) ? (uc - ukm) * g.dzi : (ukp - uc) * g.dzi;
        const float visc = nu * (uim - 2.0f * uc + uip) * g.dxi * g.dxi +
                           nu * (ujm - 2.0f * uc + ujp) * g.dyi * g.dyi +
                           nu * (ukm - 2.0f * uc + ukp) * g.dzi * g.dzi;
        const float adv = -uc * dudx - v_here * dudy - w_here * dudz;
        us[id] = uc + g.dt * (visc + adv + g.gx);
    }
    if (j >= 2) {  // advect_v_kernel, voftrial1.cu:287-342
        const float u_here = 0.25f * (__ldg(u + id - sy) + __ldg(u + id) +
                                      __ldg(u + id + 1 - sy) + __ldg(u + id + 1));
        const float w_here = 0.25f * (__ldg(w + id - sy + sz) + __ldg(w + id - sy) +
                                      __ldg(w + id) + __ldg(w + id + sz));
        const float vc = __ldg(v + id);
        const float vim = __ldg(v + id - 1), vip = __ldg(v + id + 1);
        const float vjm = __ldg(v + id - sy), vjp = __ldg(v + id + sy);
        const float vkm = __ldg(v + id - sz), vkp = __ldg(v + id + sz);
        const float dvdx = (u_here > 0.0f) ? (vc - vim) * g.dxi : (vip - vc) * g.dxi;
        const float dvdy = (vc > 0.0f) ? (vc - vjm) * g.dyi : (vjp - vc) * g.dyi;
        const float dvdz = (w_here > 0.0f) ? (vc - vkm) * g.dzi : (vkp - vc) * g.dzi;
        const float visc = nu * (vim - 2.0f * vc + vip) * g.dxi * g.dxi +
                           nu * (vjm - 2.0f * vc + vjp) * g.dyi * g.dyi +
                           nu * (vkm - 2.0f * vc + vkp) * g.dzi * g.dzi;
        const float adv = -u_here * dvdx - vc * dvdy - w_here * dvdz;
        vs[id] = vc + g.dt * (visc + adv + g.gy);
    }
    if (k >= 2) {  // advect_w_kernel, voftrial1.cu:344-399
        const float u_here = 0.25f * (__ldg(u + id + 1 - sz) + __ldg(u + id - sz) +
                                      __ldg(u + id + 1) + __ldg(u + id));
        const float v_here = 0.25f * (__ldg(v + id + sy - sz) + __ldg(v + id - sz) +
                                      __ldg(v + id) + __ldg(v + id + sy));
        const float wc = __ldg(w + id);
        const float wim = __ldg(w + id - 1), wip = __ldg(w + id + 1);
        const float wjm = __ldg(w + id - sy), wjp = __ldg(w + id + sy);
        const float wkm = __ldg(w + id - sz), wkp = __ldg(w + id + sz);
        const float dwdx = (u_here > 0.0f) ? (wc - wim) * g.dxi : (wip - wc) * g.dxi;
        const float dwdy = (v_here > 0.0f) ? (wc - wjm) * g.dyi : (wjp - wc) * g.dyi;
        const float dwdz = (wc > 0.0f) ? (wc - wkm) * g.dzi : (wkp - wc) * g.dzi;
        const float visc = nu * (wim - 2.0f * wc + wip) * g.dxi * g.dxi +
                           nu * (wjm - 2.0f * wc + wjp) * g.dyi * g.dyi +
                           nu * (wkm - 2.0f * wc + wkp) * g.dzi * g.dzi;
        const float adv = -u_here * dwdx - v_here * dwdy - wc * dwdz;
        ws[id] = wc + g.dt * (visc + adv + g.gz);
    }
}

// ---------------------------------------------------------------------------
// Pressure right-hand side rho/dt * div(u*) (voftrial1.cu:418-422).  Without
// FMA contraction the stored value is exactly the one the reference forms
// inside every Jacobi sweep, so computing it once per step changes nothing.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_rhs(Geom g,
                                             const float* __restrict__ F,
                                             const float* __restrict__ us,
                                             const float* __restrict__ vs,
                                             const float* __restrict__ ws,
                                             float* __restrict__ rhs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const int id = gidx(g, i, j, k);
    const float rho = rho_of(g, __ldg(F + id));
    rhs[id] = rho / g.dt *
              ((__ldg(us + id + 1) - __ldg(us + id)) * g.dxi +
               (__ldg(vs + id + g.px) - __ldg(vs + id)) * g.dyi +
               (__ldg(ws + id + g.plane) - __ldg(ws + id)) * g.dzi);
}

// ---------------------------------------------------------------------------
// One Jacobi sweep (voftrial1.cu:424-438): constant-coefficient 7-point
// Neumann operator, coefficients dropped on wall sides, IEEE division by ap.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_jacobi(Geom g,
                                                const float* __restrict__ rhs,
                                                const float* __restrict__ p,
                                                float* __restrict__ pt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const int id = gidx(g, i, j, k);
    const float cx = g.dxi * g.dxi, cy = g.dyi * g.dyi, cz = g.dzi * g.dzi;
    const float ae = (i != g.nx) ? cx : 0.0f;
    const float aw = (i != 1) ? cx : 0.0f;
    const float an = (j != g.ny) ? cy : 0.0f;
    const float as = (j != 1) ? cy : 0.0f;
    const float af = (k != g.nz) ? cz : 0.0f;
    const float ab = (k != 1) ? cz : 0.0f;
    const float ap = -(ae + aw + an + as + af + ab);
    pt[id] = (__ldg(rhs + id)
              - ae * __ldg(p + id + 1)
              - aw * __ldg(p + id - 1)
              - an * __ldg(p + id + g.px)
              - as * __ldg(p + id - g.px)
              - af * __ldg(p + id + g.plane)
              - ab * __ldg(p + id - g.plane)) / ap;
}

// ---------------------------------------------------------------------------
// Velocity correction fused with the free-slip boundary conditions.
// The three reference BC launches (j, then i, then k; voftrial1.cu:1116-1118)
// compose to a closed form over the whole (nx+2)(ny+2)(nz+2) box, with c* the
// index clamped to the interior range and u_new the corrected face velocity:
//   u(i,j,k) = 0                         for i == 1 or i == nx+1 (wall faces)
//            = u_new(i, cj, ck)          for 2 <= i <= nx
//            = u(0, cj, ck)  (unchanged) for i == 0
//   v(i,j,k) = 0 for j == 1 or j == ny+1, v_new(ci, j, ck) for 2<=j<=ny,
//              v(ci, 0, ck) for j == 0
//   w(i,j,k) = 0 for k == 1 or k == nz+1, w_new(ci, cj, k) for 2<=k<=nz,
//              w(ci, cj, 0) for k == 0
// Entries whose source is themselves are not rewritten, so the map has no
// read/write overlap between threads.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float corrected(const Geom& g, const float* __restrict__ F,
                                           const float* __restrict__ star,
                                           const float* __restrict__ p, int id, int s,
                                           float hinv) {
    // update_{u,v,w}_kernel, voftrial1.cu:441-493
    const float r = 0.5f * (rho_of(g, __ldg(F + id)) + rho_of(g, __ldg(F + id - s)));
    return __ldg(star + id) - g.dt / r * (__ldg(p + id) - __ldg(p + id - s)) * hinv;
}

__global__ void __launch_bounds__(256) k_correct(Geom g,
                                                 const float* __restrict__ F,
                                                 const float* __restrict__ us,
                                                 const float* __restrict__ vs,
                                                 const float* __restrict__ ws,
                                                 const float* __restrict__ p,
                                                 float* u, float* v, float* w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.nx + 1 || j > g.ny + 1 || k > g.nz + 1) return;
    const int ci = clampi(i, 1, g.nx), cj = clampi(j, 1, g.ny), ck = clampi(k, 1, g.nz);
    const int id = gidx(g, i, j, k);
    const bool jk_interior = (j == cj) && (k == ck);
    const bool ik_interior = (i == ci) && (k == ck);
    const bool ij_interior = (i == ci) && (j == cj);

    // u
    if (i == 1 || i == g.nx + 1) {
        u[id] = 0.0f;
    } else if (i >= 2) {
        u[id] = corrected(g, F, us, p, gidx(g, i, cj, ck), 1, g.dxi);
    } else if (!jk_interior) {  // i == 0: stale column, ghost copy
        u[id] = u[gidx(g, 0, cj, ck)];
    }
    // v
    if (j == 1 || j == g.ny + 1) {
        v[id] = 0.0f;
    } else if (j >= 2) {
        v[id] = corrected(g, F, vs, p, gidx(g, ci, j, ck), g.px, g.dyi);
    } else if (!ik_interior) {
        v[id] = v[gidx(g, ci, 0, ck)];
    }
    // w
    if (k == 1 || k == g.nz + 1) {
        w[id] = 0.0f;
    } else if (k >= 2) {
        w[id] = corrected(g, F, ws, p, gidx(g, ci, cj, k), g.plane, g.dzi);
    } else if (!ij_interior) {
        w[id] = w[gidx(g, ci, cj, 0)];
    }
}

// ---------------------------------------------------------------------------
// One FCT sweep along AXIS (0=x, 1=y, 2=z), stages 1-4 fused.
//
// Along one grid line the four reference stages only couple cells of that
// line: the other direction's antidiffusive fluxes are zeroed by stage 2 of
// the same sweep (voftrial1.cu:573-574, 712-713), so their terms in pp, pm and
// stage 4 vanish (exactly, up to the sign of a zero that clamp01f removes).
// A block therefore loads TL whole lines (cells 0..n+1) into shared memory and
// runs the stages there.  Conventions reproduced from the reference's
// never-written, zero-filled buffers (voftrial1.cu:1200-1203):
//   Ftd at the line's ghost cells is 0, rp/rm at ghost cells are 0, and the
//   limiter of the first face (c[1]) is 0.
// Q2 length factors per sweep (x / y / z):
//   stage 1 flux term  (f_l - f_r)*dy*dz/vol | (f_l - f_r)*dy/(dx*dy) | (f_l - f_r)*dy*dx/vol
//   dv factor          dt*dy*dz              | dt*dx*dz               | dt*dx*dy
//   limiter q          *dx                   | *dx                    | *dz
//   stage 4 divisor    /dy                   | /dy                    | /dz
// FINAL: last sweep of the step; also applies post_process_f_kernel (a second
// clamp01f) and apply_bc_F (ghost = value at the clamped interior index).
// ---------------------------------------------------------------------------
constexpr int FCT_TL = 16;            // lines per tile
constexpr int FCT_LP = FCT_TL + 1;    // padded line pitch in shared memory
constexpr int FCT_THREADS = 256;

template <int AXIS>
struct LineMap {
    // Line coordinates (a, b) = the two other axes; position q along AXIS.
    __device__ static int n(const Geom& g) { return AXIS == 0 ? g.nx : (AXIS == 1 ? g.ny : g.nz); }
    __device__ static int na(const Geom& g) { return AXIS == 0 ? g.ny : g.nx; }
    __device__ static int nb(const Geom& g) { return AXIS == 2 ? g.ny : g.nz; }
    __device__ static int stride(const Geom& g) { return AXIS == 0 ? 1 : (AXIS == 1 ? g.px : g.plane); }
    __device__ static int base(const Geom& g, int a, int b) {
        // a: y for AXIS 0, x otherwise; b: z for AXIS 0/1, y for AXIS 2
        if (AXIS == 0) return gidx(g, 0, a, b);
        if (AXIS == 1) return gidx(g, a, 0, b);
        return gidx(g, a, b, 0);
    }
};

template <int AXIS, bool FINAL>
__global__ void __launch_bounds__(FCT_THREADS) k_fct(Geom g, float* F, const float* __restrict__ vel) {
    extern __shared__ float smem[];
    using M = LineMap<AXIS>;
    const int n = M::n(g);
    const int np = n + 2;                 // positions 0..n+1
    float* sF = smem;                     // F, later reused for rp
    float* sV = sF + np * FCT_LP;         // face velocity (positions 1..n+1)
    float* sT = sV + np * FCT_LP;         // Ftd
    float* sA = sT + np * FCT_LP;         // antidiffusive flux a[f] (faces 1..n+1)
    float* sM = sA + np * FCT_LP;         // rm

    const int a0 = 1 + blockIdx.x * FCT_TL;   // first line coordinate a of this tile
    const int b = 1 + blockIdx.y;             // line coordinate b
    const int nl = min(FCT_TL, M::na(g) - a0 + 1);
    const int lstride = (AXIS == 0) ? g.px : 1;   // global distance between adjacent lines
    const int qs = M::stride(g);
    const int gbase = M::base(g, a0, b);
    const int total = np * FCT_TL;

    // Thread -> (q, l) mapping: position-fastest for x lines (contiguous in
    // memory along q), line-fastest for y/z tiles (contiguous along a).
    auto qof = [&](int t) { return AXIS == 0 ? (t % np) : (t / FCT_TL); };
    auto lof = [&](int t) { return AXIS == 0 ? (t / np) : (t % FCT_TL); };

    // ---- load F (positions 0..n+1) and the face velocity (1..n+1) ----
    for (int t = threadIdx.x; t < total; t += FCT_THREADS) {
        const int q = qof(t), l = lof(t);
        if (l < nl) {
            const int gi = gbase + l * lstride + q * qs;
            sF[q * FCT_LP + l] = F[gi];
            if (q >= 1) sV[q * FCT_LP + l] = __ldg(vel + gi);
        }
    }
    __syncthreads();

    const float dt = g.dt;
    const float vol = g.dx * g.dy * g.dz;
    const float dvfac = (AXIS == 0) ? dt * g.dy * g.dz : (AXIS == 1 ? dt * g.dx * g.dz : dt * g.dx * g.dy);
    const float hq = (AXIS == 2) ? g.dz : g.dx;
    const float h4 = (AXIS == 2) ? g.dz : g.dy;

    // Low-order (donor) and high-order fluxes through face f (between cells
    // f-1 and f), as fl_L / fl_H of fct_*_stage1/2.
    auto flux_low = [&](int f, int l) {
        const float uf = sV[f * FCT_LP + l];
        return (uf >= 0.0f) ? uf * dt * sF[(f - 1) * FCT_LP + l] : uf * dt * sF[f * FCT_LP + l];
    };
    auto flux_high = [&](int f, int l) {
        const float uf = sV[f * FCT_LP + l];
        return (uf <= 0.0f) ? uf * dt * sF[(f - 1) * FCT_LP + l] : uf * dt * sF[f * FCT_LP + l];
    };

    // ---- stage 1 (Ftd) and the antidiffusive face fluxes (stage 2, first half) ----
    for (int t = threadIdx.x; t < total; t += FCT_THREADS) {
        const int q = qof(t), l = lof(t);
        if (l >= nl) continue;
        if (q >= 1 && q <= n) {
            const float fl = flux_low(q, l);
            const float fr = flux_low(q + 1, l);
            const float dv = vol - dvfac * (sV[(q + 1) * FCT_LP + l] - sV[q * FCT_LP + l]);
            float term;
            if (AXIS == 0) term = (fl - fr) * g.dy * g.dz / vol;
            else if (AXIS == 1) term = (fl - fr) * g.dy / (g.dx * g.dy);
            else term = (fl - fr) * g.dy * g.dx / vol;
            float out = (sF[q * FCT_LP + l] + term) * vol / dv;
            if (out > 1.0f || out < 0.0f) out = clamp01f(out);
            sT[q * FCT_LP + l] = out;
        } else {
            sT[q * FCT_LP + l] = 0.0f;  // Ftd ghost cells are never written
        }
        if (q >= 1) sA[q * FCT_LP + l] = flux_high(q, l) - flux_low(q, l);
    }
    __syncthreads();

    // ---- stage 2 (second half): Zalesak ratios rp (into sF) and rm ----
    for (int t = threadIdx.x; t < total; t += FCT_THREADS) {
        const int q = qof(t), l = lof(t);
        if (l >= nl) continue;
        float rp = 0.0f, rm = 0.0f;  // ghost cells keep 0
        if (q >= 1 && q <= n) {
            const float tc = sT[q * FCT_LP + l];
            const float tm = sT[(q - 1) * FCT_LP + l];
            const float tp = sT[(q + 1) * FCT_LP + l];
            const float fmx = fmaxf(tc, fmaxf(tm, tp));
            const float fmn = fminf(tc, fminf(tm, tp));
            const float al = sA[q * FCT_LP + l];
            const float ar = sA[(q + 1) * FCT_LP + l];
            const float pp = fmaxf(0.0f, al) - fminf(0.0f, ar);
            const float qp = (fmx - tc) * hq;
            rp = (pp > 0.0f) ? fminf(1.0f, qp / pp) : 0.0f;
            const float pm = fmaxf(0.0f, ar) - fminf(0.0f, al);
            const float qm = (tc - fmn) * hq;
            rm = (pm > 0.0f) ? fminf(1.0f, qm / pm) : 0.0f;
        }
        sF[q * FCT_LP + l] = rp;
        sM[q * FCT_LP + l] = rm;
    }
    __syncthreads();

    // ---- stage 3 (face limiter) + stage 4 (antidiffusive correction) ----
    const int na = M::na(g), nb = M::nb(g);
    for (int t = threadIdx.x; t < total; t += FCT_THREADS) {
        const int q = qof(t), l = lof(t);
        if (l >= nl || q < 1 || q > n) continue;
        // c[f] = limiter of face f (stage 3); c[1] is never written -> 0.
        auto climit = [&](int f) {
            if (f == 1) return 0.0f;
            const float af = sA[f * FCT_LP + l];
            return (af >= 0.0f) ? fminf(sF[f * FCT_LP + l], sM[(f - 1) * FCT_LP + l])
                                : fminf(sF[(f - 1) * FCT_LP + l], sM[f * FCT_LP + l]);
        };
        const float cl = climit(q);
        const float cr = climit(q + 1);
        const float al = sA[q * FCT_LP + l];
        const float ar = sA[(q + 1) * FCT_LP + l];
        const float dv = vol - dvfac * (sV[(q + 1) * FCT_LP + l] - sV[q * FCT_LP + l]);
        const float out = sT[q * FCT_LP + l] - ((ar * cr - al * cl) / h4) * vol / dv;
        float fnew = clamp01f(out);
        const int a = a0 + l;
        const int gi = gbase + l * lstride + q * qs;
        if (!FINAL) {
            F[gi] = fnew;
        } else {
            fnew = clamp01f(fnew);  // post_process_f_kernel, voftrial1.cu:502-507
            // apply_bc_F (voftrial1.cu:1122-1135): every ghost cell takes the
            // value at its clamped interior index.  This thread owns the
            // interior cell (q, a, b) and writes every cell that maps onto it.
            int qv[3], av[3], bv[3];
            int nq = 0, nav = 0, nbv = 0;
            qv[nq++] = q;
            if (q == 1) qv[nq++] = 0;
            if (q == n) qv[nq++] = n + 1;
            av[nav++] = a;
            if (a == 1) av[nav++] = 0;
            if (a == na) av[nav++] = na + 1;
            bv[nbv++] = b;
            if (b == 1) bv[nbv++] = 0;
            if (b == nb) bv[nbv++] = nb + 1;
            for (int ib = 0; ib < nbv; ++ib)
                for (int ia = 0; ia < nav; ++ia) {
                    const int lb = M::base(g, av[ia], bv[ib]);
                    for (int iq = 0; iq < nq; ++iq) F[lb + qv[iq] * qs] = fnew;
                }
        }
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static inline dim3 interior_grid(const Geom& g, dim3 blk) {
    return dim3((g.nx + blk.x - 1) / blk.x, (g.ny + blk.y - 1) / blk.y, (g.nz + blk.z - 1) / blk.z);
}

size_t fct_smem_bytes(int n) { return sizeof(float) * 5u * (size_t)(n + 2) * FCT_LP; }

template <int AXIS, bool FINAL>
static cudaError_t launch_fct(const Geom& g, float* F, const float* vel, cudaStream_t s) {
    const int n = AXIS == 0 ? g.nx : (AXIS == 1 ? g.ny : g.nz);
    const int na = AXIS == 0 ? g.ny : g.nx;
    const int nb = AXIS == 2 ? g.ny : g.nz;
    const size_t smem = fct_smem_bytes(n);
    dim3 grid((na + FCT_TL - 1) / FCT_TL, nb, 1);
    k_fct<AXIS, FINAL><<<grid, FCT_THREADS, smem, s>>>(g, F, vel);
    return cudaGetLastError();
}

cudaError_t plain_configure(int max_line) {
    // The attribute is a per-function ceiling shared by every context on the
    // device, so it is raised to the device's opt-in maximum rather than to
    // this grid's need (a later, smaller grid must not lower it).
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    if (fct_smem_bytes(max_line) > (size_t)optin) return cudaErrorInvalidValue;
    const size_t smem = (size_t)optin;
#define VOF_SET_SMEM(A, FIN)                                                              \
    e = cudaFuncSetAttribute(k_fct<A, FIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                             (int)smem);                                                  \
    if (e != cudaSuccess) return e;
    VOF_SET_SMEM(0, false) VOF_SET_SMEM(0, true)
    VOF_SET_SMEM(1, false) VOF_SET_SMEM(1, true)
    VOF_SET_SMEM(2, false) VOF_SET_SMEM(2, true)
#undef VOF_SET_SMEM
    return cudaSuccess;
}

bool plain_supported(const Geom& g) {
    const int m = g.nx > g.ny ? (g.nx > g.nz ? g.nx : g.nz) : (g.ny > g.nz ? g.ny : g.nz);
    return fct_smem_bytes(m) <= 227u * 1024u;
}

int plain_kernels_per_step(int jacobi_iters) { return 1 + 1 + jacobi_iters + 1 + 3; }

cudaError_t plain_step(const Geom& g, const PlainBuffers& b, int istep, int jacobi_iters,
                       int* p_parity, cudaStream_t s, cudaEvent_t* ev) {
    const dim3 blk(32, 4, 2);
    const dim3 grid = interior_grid(g, blk);
    cudaError_t e;
    // ev (optional, PLAIN_PHASES+1 events): ev[0] before the step, ev[q+1]
    // after phase q (predict, rhs, jacobi, correct, sweep 1, sweep 2, sweep 3).
    auto mark = [&](int q) -> cudaError_t { return ev ? cudaEventRecord(ev[q], s) : cudaSuccess; };

    if ((e = mark(0)) != cudaSuccess) return e;
    k_predict<<<grid, blk, 0, s>>>(g, b.F, b.u, b.v, b.w, b.us, b.vs, b.ws);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = mark(1)) != cudaSuccess) return e;
    k_rhs<<<grid, blk, 0, s>>>(g, b.F, b.us, b.vs, b.ws, b.rhs);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = mark(2)) != cudaSuccess) return e;

    // Jacobi ping-pong (voftrial1.cu:1371-1375); *p_parity says which of the
    // two pressure buffers holds the current iterate.
    float* pbuf[2] = {b.p0, b.p1};
    int cur = *p_parity;
    for (int it = 0; it < jacobi_iters; ++it) {
        k_jacobi<<<grid, blk, 0, s>>>(g, b.rhs, pbuf[cur], pbuf[cur ^ 1]);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        cur ^= 1;
    }
    *p_parity = cur;
    if ((e = mark(3)) != cudaSuccess) return e;

    const dim3 gfull((g.nx + 2 + blk.x - 1) / blk.x, (g.ny + 2 + blk.y - 1) / blk.y,
                     (g.nz + 2 + blk.z - 1) / blk.z);
    k_correct<<<gfull, blk, 0, s>>>(g, b.F, b.us, b.vs, b.ws, pbuf[cur], b.u, b.v, b.w);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = mark(4)) != cudaSuccess) return e;

    // Sweep order by istep % 3 (voftrial1.cu:1384-1396).
    const int r = ((istep % 3) + 3) % 3;
    static const int order[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
    for (int q = 0; q < 3; ++q) {
        const int axis = order[r][q];
        const bool last = (q == 2);
        const float* vel = axis == 0 ? b.u : (axis == 1 ? b.v : b.w);
        if (axis == 0) e = last ? launch_fct<0, true>(g, b.F, vel, s) : launch_fct<0, false>(g, b.F, vel, s);
        else if (axis == 1) e = last ? launch_fct<1, true>(g, b.F, vel, s) : launch_fct<1, false>(g, b.F, vel, s);
        else e = last ? launch_fct<2, true>(g, b.F, vel, s) : launch_fct<2, false>(g, b.F, vel, s);
        if (e != cudaSuccess || (e = mark(5 + q)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int plain_phase_launches(int phase, int jacobi_iters) {
    return phase == PHASE_JACOBI ? jacobi_iters : 1;
}

}  // namespace vof
