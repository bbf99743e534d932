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
//   k_predict2     advect_{u,v,w}_kernel + cal_nu_rho_kernel   voftrial1.cu:95-104, 230-399
//                  two cells per thread (k_predict: one; VOF_PREDICT=1)
//   k_rhs4         the rhs expression of solve_p_jacobi_kernel voftrial1.cu:418-422
//                  four cells per thread (k_rhs: one, marching z; VOF_RHS=1)
//   k_jacobi_peel  (jacobi_tb.cu) one solve_p_jacobi_kernel sweep per launch,  voftrial1.cu:401-439
//                  two cells per thread (alternatives selected by VOF_JACOBI, below)
//   k_correct4     update_{u,v,w}_kernel + apply_bc_velocity   voftrial1.cu:441-493, 959-1051, 1107-1120
//                  four cells per thread (k_correct: one; VOF_CORRECT=1)
//   k_fct<AXIS,FINAL>  (fct_sweep.cu) fct_{x,y,z}_sweep_stage1..4, and on
//                  the last sweep post_process_f_kernel + apply_bc_F   voftrial1.cu:502-905, 1053-1135
#include "plain_step.h"

#include "fct_sweep.h"
#include "jacobi_tb.h"

#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

namespace vof {

#ifndef VOF_PLAIN_NO_FMAD_CHECK
// Compile-time guard: the build must pass -fmad=false for this file.
#if defined(__CUDA_ARCH__) && !defined(VOF_FMAD_FALSE)
#error "plain_step.cu must be compiled with -fmad=false -DVOF_FMAD_FALSE"
#endif
#endif

// All kernels below march along z: a thread owns one (i, j) column of a
// 32 x 8 tile and walks a chunk of k, computing its index once and carrying
// the column's k-1 / k / k+1 values in registers; in-plane neighbours come
// from L1.  The per-point arithmetic is the reference's, unchanged.
constexpr int TX = 32, TY = 8;

struct Column {
    int i, j, k0, k1;
    __device__ Column(const Geom& g, int lo_i, int lo_j, int kchunk) {
        i = blockIdx.x * TX + threadIdx.x + lo_i;
        j = blockIdx.y * TY + threadIdx.y + lo_j;
        k0 = 1 + blockIdx.z * kchunk;
        k1 = min(g.nz, k0 + kchunk - 1);
    }
};

// Indices whose clamped value is x on an axis of n interior cells: x itself,
// plus the ghost 0 when x == 1 and the ghost n+1 when x == n.
__device__ __forceinline__ int mirrors(int x, int n, int* out) {
    // fixed positions (no runtime index: the list stays in registers)
    out[0] = x;
    out[1] = (x == 1) ? 0 : n + 1;
    out[2] = n + 1;
    return 1 + (x == 1) + (x == n);
}

// ---------------------------------------------------------------------------
// Momentum predictor: u*, v*, w* on the interior faces the reference updates
// (u: i in [imin+1, imax], j,k interior; v, w likewise), nu from F on the fly.
// advect_u/v/w_kernel + cal_nu_rho_kernel, voftrial1.cu:95-104, 230-399.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_predict(Geom g,
                                                 const float* __restrict__ F,
                                                 const float* __restrict__ u,
                                                 const float* __restrict__ v,
                                                 const float* __restrict__ w,
                                                 float* __restrict__ us,
                                                 float* __restrict__ vs,
                                                 float* __restrict__ ws, int kchunk) {
    const Column col(g, 1, 1, kchunk);
    const int i = col.i, j = col.j;
    if (i > g.nx || j > g.ny || col.k0 > g.nz) return;
    const int sy = g.px, sz = g.plane;
    int id = gidx(g, i, j, col.k0);
    // column windows along k
    float u_km = __ldg(u + id - sz), u_c = __ldg(u + id);
    float v_km = __ldg(v + id - sz), v_c = __ldg(v + id);
    float w_km = __ldg(w + id - sz), w_c = __ldg(w + id);
    float wim_c = __ldg(w + id - 1), wjm_c = __ldg(w + id - sy);
    float uip_km = __ldg(u + id + 1 - sz), vjp_km = __ldg(v + id + sy - sz);
    for (int k = col.k0; k <= col.k1; ++k, id += sz) {
        const float u_kp = __ldg(u + id + sz), v_kp = __ldg(v + id + sz), w_kp = __ldg(w + id + sz);
        const float wim_kp = __ldg(w + id - 1 + sz), wjm_kp = __ldg(w + id - sy + sz);
        const float uip_c = __ldg(u + id + 1), vjp_c = __ldg(v + id + sy);
        const float nu = nu_of(g, __ldg(F + id));

        if (i >= 2) {  // advect_u_kernel, voftrial1.cu:230-285
            const float v_here = 0.25f * (__ldg(v + id - 1) + __ldg(v + id - 1 + sy) + v_c + vjp_c);
            const float w_here = 0.25f * (wim_c + wim_kp + w_c + w_kp);
            const float uim = __ldg(u + id - 1);
            const float ujm = __ldg(u + id - sy), ujp = __ldg(u + id + sy);
            const float dudx = (u_c > 0.0f) ? (u_c - uim) * g.dxi : (uip_c - u_c) * g.dxi;
            const float dudy = (v_here > 0.0f) ? (u_c - ujm) * g.dyi : (ujp - u_c) * g.dyi;
            const float dudz = (w_here > 0.0f) ? (u_c - u_km) * g.dzi : (u_kp - u_c) * g.dzi;
            const float visc = nu * (uim - 2.0f * u_c + uip_c) * g.dxi * g.dxi +
                               nu * (ujm - 2.0f * u_c + ujp) * g.dyi * g.dyi +
                               nu * (u_km - 2.0f * u_c + u_kp) * g.dzi * g.dzi;
            const float adv = -u_c * dudx - v_here * dudy - w_here * dudz;
            us[id] = u_c + g.dt * (visc + adv + g.gx);
        }
        if (j >= 2) {  // advect_v_kernel, voftrial1.cu:287-342
            const float u_here = 0.25f * (__ldg(u + id - sy) + u_c + __ldg(u + id + 1 - sy) + uip_c);
            const float w_here = 0.25f * (wjm_kp + wjm_c + w_c + w_kp);
            const float vim = __ldg(v + id - 1), vip = __ldg(v + id + 1);
            const float vjm = __ldg(v + id - sy);
            const float dvdx = (u_here > 0.0f) ? (v_c - vim) * g.dxi : (vip - v_c) * g.dxi;
            const float dvdy = (v_c > 0.0f) ? (v_c - vjm) * g.dyi : (vjp_c - v_c) * g.dyi;
            const float dvdz = (w_here > 0.0f) ? (v_c - v_km) * g.dzi : (v_kp - v_c) * g.dzi;
            const float visc = nu * (vim - 2.0f * v_c + vip) * g.dxi * g.dxi +
                               nu * (vjm - 2.0f * v_c + vjp_c) * g.dyi * g.dyi +
                               nu * (v_km - 2.0f * v_c + v_kp) * g.dzi * g.dzi;
            const float adv = -u_here * dvdx - v_c * dvdy - w_here * dvdz;
            vs[id] = v_c + g.dt * (visc + adv + g.gy);
        }
        if (k >= 2) {  // advect_w_kernel, voftrial1.cu:344-399
            const float u_here = 0.25f * (uip_km + u_km + uip_c + u_c);
            const float v_here = 0.25f * (vjp_km + v_km + v_c + vjp_c);
            const float wip = __ldg(w + id + 1), wjp = __ldg(w + id + sy);
            const float dwdx = (u_here > 0.0f) ? (w_c - wim_c) * g.dxi : (wip - w_c) * g.dxi;
            const float dwdy = (v_here > 0.0f) ? (w_c - wjm_c) * g.dyi : (wjp - w_c) * g.dyi;
            const float dwdz = (w_c > 0.0f) ? (w_c - w_km) * g.dzi : (w_kp - w_c) * g.dzi;
            const float visc = nu * (wim_c - 2.0f * w_c + wip) * g.dxi * g.dxi +
                               nu * (wjm_c - 2.0f * w_c + wjp) * g.dyi * g.dyi +
                               nu * (w_km - 2.0f * w_c + w_kp) * g.dzi * g.dzi;
            const float adv = -u_here * dwdx - v_here * dwdy - w_c * dwdz;
            ws[id] = w_c + g.dt * (visc + adv + g.gz);
        }
        u_km = u_c; u_c = u_kp;
        v_km = v_c; v_c = v_kp;
        w_km = w_c; w_c = w_kp;
        wim_c = wim_kp; wjm_c = wjm_kp;
        uip_km = uip_c; vjp_km = vjp_c;
    }
}

// The predictor with two cells per thread.  Cells are paired by padded column
// (2m, 2m + 1: one aligned 8-byte word), the pairs of all rows of a plane
// numbered flat so that 32 consecutive pairs make a warp across row ends, and
// a thread marches a chunk of planes, carrying its pair's k-1 / k values in
// registers as k_predict does.  Every operand is a float2 load (10 per pair
// and plane: u, v, w of the next plane, the rows j-1 and j+1 of u, v, w,
// w of the next plane's row j-1, v of row j+1, and F); the x-1 and x+1
// neighbours come from the lanes beside (a pair's left neighbour is the left
// lane's second cell, its right neighbour the right lane's first), or from
// memory at the ends of a warp and of a row.  Each cell's three updates keep
// k_predict's expressions and operand order (same bits).
// The pair's left (x-1 of the first cell) and right (x+1 of the second cell)
// neighbours of a value held as a pair by every lane.
__device__ __forceinline__ float left_of(float2 a, bool ldw, const float* __restrict__ p, int idl) {
    const float s = __shfl_up_sync(0xffffffffu, a.y, 1);
    return ldw ? __ldg(p + idl) : s;
}
__device__ __forceinline__ float right_of(float2 a, bool lde, const float* __restrict__ p, int idr) {
    const float s = __shfl_down_sync(0xffffffffu, a.x, 1);
    return lde ? __ldg(p + idr) : s;
}

__global__ void __launch_bounds__(256, 4) k_predict2(Geom g, const float* __restrict__ F,
                                                     const float* __restrict__ u, const float* __restrict__ v,
                                                     const float* __restrict__ w, float* __restrict__ us,
                                                     float* __restrict__ vs, float* __restrict__ ws, int kchunk) {
    const int npair = g.nx / 2 + 1;  // pairs covering columns 0 .. nx
    const int nq = npair * g.ny;
    const int qt = blockIdx.x * blockDim.x + threadIdx.x;
    const bool qa = qt < nq;
    const int q = qa ? qt : nq - 1;  // lanes past the end shadow the last pair
    const int jr = q / npair, m = q - jr * npair;
    const int j = jr + 1, i0 = 2 * m;
    const int lane = threadIdx.x & 31;
    const bool ldw = lane == 0 && m > 0;            // x-1 neighbours from memory
    const bool lde = lane == 31 || m == npair - 1;  // x+1 neighbours from memory
    const int k0 = 1 + blockIdx.y * kchunk, k1 = min(g.nz, k0 + kchunk - 1);
    const int sy = g.px, sz = g.plane;
    // which cells of the pair are updated (u from i = 2, v and w from i = 1)
    const bool a0 = qa && i0 >= 1 && i0 <= g.nx, a1 = qa && i0 + 1 <= g.nx;
    const bool u0 = qa && i0 >= 2 && i0 <= g.nx, u1 = qa && i0 + 1 >= 2 && i0 + 1 <= g.nx;
    auto L2 = [](const float* __restrict__ p, int id) { return __ldg(reinterpret_cast<const float2*>(p + id)); };
    int id = gidx(g, i0, j, k0);  // even
    // column windows along k (values of the pair's two cells)
    float2 u_km = L2(u, id - sz), u_c = L2(u, id);
    float2 v_km = L2(v, id - sz), v_c = L2(v, id);
    float2 w_km = L2(w, id - sz), w_c = L2(w, id);
    float2 wjm_c = L2(w, id - sy), vjp_km = L2(v, id + sy - sz);
    // x neighbours carried from the previous plane
    float wim_c = left_of(w_c, ldw, w, id - 1);
    float uip_km = right_of(u_km, lde, u, id + 2 - sz);
    for (int k = k0; k <= k1; ++k, id += sz) {
        const float2 u_kp = L2(u, id + sz), v_kp = L2(v, id + sz), w_kp = L2(w, id + sz);
        const float2 wjm_kp = L2(w, id - sy + sz), vjp_c = L2(v, id + sy);
        const float2 ujm = L2(u, id - sy), ujp = L2(u, id + sy), vjm = L2(v, id - sy), wjp = L2(w, id + sy);
        const float2 f2 = L2(F, id);
        const float wim_kp = left_of(w_kp, ldw, w, id - 1 + sz);
        const float uim0 = left_of(u_c, ldw, u, id - 1), uip1 = right_of(u_c, lde, u, id + 2);
        const float vim0 = left_of(v_c, ldw, v, id - 1), vip1 = right_of(v_c, lde, v, id + 2);
        const float vjp_im0 = left_of(vjp_c, ldw, v, id - 1 + sy);
        const float ujm_ip1 = right_of(ujm, lde, u, id + 2 - sy);
        const float wip1 = right_of(w_c, lde, w, id + 2);
        float out_u[2], out_v[2], out_w[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            // this cell's values and its x neighbours
            const float uc = e ? u_c.y : u_c.x, ukm = e ? u_km.y : u_km.x, ukp = e ? u_kp.y : u_kp.x;
            const float vc = e ? v_c.y : v_c.x, vkm = e ? v_km.y : v_km.x, vkp = e ? v_kp.y : v_kp.x;
            const float wc = e ? w_c.y : w_c.x, wkm = e ? w_km.y : w_km.x, wkp = e ? w_kp.y : w_kp.x;
            const float uim = e ? u_c.x : uim0, uip_c = e ? uip1 : u_c.y;
            const float vim = e ? v_c.x : vim0, vip = e ? vip1 : v_c.y;
            const float wim_cc = e ? w_c.x : wim_c, wim_kpp = e ? w_kp.x : wim_kp;
            const float wip = e ? wip1 : w_c.y;
            const float vjpc = e ? vjp_c.y : vjp_c.x, vjp_im = e ? vjp_c.x : vjp_im0;
            const float vjpkm = e ? vjp_km.y : vjp_km.x;
            const float ujmc = e ? ujm.y : ujm.x, ujpc = e ? ujp.y : ujp.x, ujm_ip = e ? ujm_ip1 : ujm.y;
            const float vjmc = e ? vjm.y : vjm.x;
            const float wjmc = e ? wjm_c.y : wjm_c.x, wjmkp = e ? wjm_kp.y : wjm_kp.x;
            const float wjpc = e ? wjp.y : wjp.x;
            const float uipkm = e ? uip_km : u_km.y;
            const float nu = nu_of(g, e ? f2.y : f2.x);
            {  // advect_u_kernel, voftrial1.cu:230-285
                const float v_here = 0.25f * (vim + vjp_im + vc + vjpc);
                const float w_here = 0.25f * (wim_cc + wim_kpp + wc + wkp);
                const float dudx = (uc > 0.0f) ? (uc - uim) * g.dxi : (uip_c - uc) * g.dxi;
                const float dudy = (v_here > 0.0f) ? (uc - ujmc) * g.dyi : (ujpc - uc) * g.dyi;
                const float dudz = (w_here > 0.0f) ? (uc - ukm) * g.dzi : (ukp - uc) * g.dzi;
                const float visc = nu * (uim - 2.0f * uc + uip_c) * g.dxi * g.dxi +
                                   nu * (ujmc - 2.0f * uc + ujpc) * g.dyi * g.dyi +
                                   nu * (ukm - 2.0f * uc + ukp) * g.dzi * g.dzi;
                const float adv = -uc * dudx - v_here * dudy - w_here * dudz;
                out_u[e] = uc + g.dt * (visc + adv + g.gx);
            }
            {  // advect_v_kernel, voftrial1.cu:287-342
                const float u_here = 0.25f * (ujmc + uc + ujm_ip + uip_c);
                const float w_here = 0.25f * (wjmkp + wjmc + wc + wkp);
                const float dvdx = (u_here > 0.0f) ? (vc - vim) * g.dxi : (vip - vc) * g.dxi;
                const float dvdy = (vc > 0.0f) ? (vc - vjmc) * g.dyi : (vjpc - vc) * g.dyi;
                const float dvdz = (w_here > 0.0f) ? (vc - vkm) * g.dzi : (vkp - vc) * g.dzi;
                const float visc = nu * (vim - 2.0f * vc + vip) * g.dxi * g.dxi +
                                   nu * (vjmc - 2.0f * vc + vjpc) * g.dyi * g.dyi +
                                   nu * (vkm - 2.0f * vc + vkp) * g.dzi * g.dzi;
                const float adv = -u_here * dvdx - vc * dvdy - w_here * dvdz;
                out_v[e] = vc + g.dt * (visc + adv + g.gy);
            }
            {  // advect_w_kernel, voftrial1.cu:344-399
                const float u_here = 0.25f * (uipkm + ukm + uip_c + uc);
                const float v_here = 0.25f * (vjpkm + vkm + vc + vjpc);
                const float dwdx = (u_here > 0.0f) ? (wc - wim_cc) * g.dxi : (wip - wc) * g.dxi;
                const float dwdy = (v_here > 0.0f) ? (wc - wjmc) * g.dyi : (wjpc - wc) * g.dyi;
                const float dwdz = (wc > 0.0f) ? (wc - wkm) * g.dzi : (wkp - wc) * g.dzi;
                const float visc = nu * (wim_cc - 2.0f * wc + wip) * g.dxi * g.dxi +
                                   nu * (wjmc - 2.0f * wc + wjpc) * g.dyi * g.dyi +
                                   nu * (wkm - 2.0f * wc + wkp) * g.dzi * g.dzi;
                const float adv = -u_here * dwdx - v_here * dwdy - wc * dwdz;
                out_w[e] = wc + g.dt * (visc + adv + g.gz);
            }
        }
        float2* US = reinterpret_cast<float2*>(us + id);
        if (u0 && u1)
            *US = make_float2(out_u[0], out_u[1]);
        else if (u0)
            us[id] = out_u[0];
        else if (u1)
            us[id + 1] = out_u[1];
        if (j >= 2) {
            if (a0 && a1)
                *reinterpret_cast<float2*>(vs + id) = make_float2(out_v[0], out_v[1]);
            else if (a0)
                vs[id] = out_v[0];
            else if (a1)
                vs[id + 1] = out_v[1];
        }
        if (k >= 2) {
            if (a0 && a1)
                *reinterpret_cast<float2*>(ws + id) = make_float2(out_w[0], out_w[1]);
            else if (a0)
                ws[id] = out_w[0];
            else if (a1)
                ws[id + 1] = out_w[1];
        }
        u_km = u_c;
        u_c = u_kp;
        v_km = v_c;
        v_c = v_kp;
        w_km = w_c;
        w_c = w_kp;
        wim_c = wim_kp;
        wjm_c = wjm_kp;
        uip_km = uip1;
        vjp_km = vjp_c;
    }
}

// ---------------------------------------------------------------------------
// Continuum surface force (extension; no counterpart in the reference, whose
// sigma no kernel reads).  J. U. Brackbill, D. B. Kothe, C. Zemach, "A
// continuum method for modeling surface tension", J. Comput. Phys. 100 (1992):
// the body force sigma kappa grad(F) with the interface normal n = grad F /
// |grad F| and kappa = -div n, both by central differences at cell centres;
// F's ghosts are the zero-gradient copies, and a normal beyond a wall is the
// mirror image of the one inside (its wall-normal component negated: a 90
// degree contact angle).  On a face, kappa is the mean of its two cells,
// grad F their difference, and the acceleration is divided by the face
// density of the correction, 0.5 (rho_a + rho_b); it is added to u*, v*, w*
// on the faces the predictor updates.  FP32, operations in a fixed order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_csf_normal(Geom g, const float* __restrict__ F, float* __restrict__ nx_,
                                                    float* __restrict__ ny_, float* __restrict__ nz_) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const int id = gidx(g, i, j, k);
    const float hx = 0.5f * g.dxi, hy = 0.5f * g.dyi, hz = 0.5f * g.dzi;
    const float gxv = (F[id + 1] - F[id - 1]) * hx;
    const float gyv = (F[id + g.px] - F[id - g.px]) * hy;
    const float gzv = (F[id + g.plane] - F[id - g.plane]) * hz;
    const float mag = sqrtf(gxv * gxv + gyv * gyv + gzv * gzv);
    const float eps = 1e-6f * g.dxi;
    const bool has = mag > eps;
    nx_[id] = has ? gxv / mag : 0.0f;
    ny_[id] = has ? gyv / mag : 0.0f;
    nz_[id] = has ? gzv / mag : 0.0f;
}

__global__ void __launch_bounds__(256) k_csf_curv(Geom g, const float* __restrict__ nx_,
                                                  const float* __restrict__ ny_, const float* __restrict__ nz_,
                                                  float* __restrict__ kap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const int id = gidx(g, i, j, k);
    const float hx = 0.5f * g.dxi, hy = 0.5f * g.dyi, hz = 0.5f * g.dzi;
    // neighbours beyond a wall: the mirror image of the cell at the wall
    const float xe = i < g.nx ? nx_[id + 1] : -nx_[id], xw = i > 1 ? nx_[id - 1] : -nx_[id];
    const float yn = j < g.ny ? ny_[id + g.px] : -ny_[id], ys = j > 1 ? ny_[id - g.px] : -ny_[id];
    const float zu = k < g.nz ? nz_[id + g.plane] : -nz_[id], zd = k > 1 ? nz_[id - g.plane] : -nz_[id];
    kap[id] = -((xe - xw) * hx + (yn - ys) * hy + (zu - zd) * hz);
}

__device__ __forceinline__ float csf_accel(const Geom& g, float Fa, float Fb, float ka, float kb, float hinv) {
    const float f = g.sigma * (0.5f * (ka + kb)) * ((Fb - Fa) * hinv);
    const float r = 0.5f * (rho_of(g, Fa) + rho_of(g, Fb));
    return f / r;
}

__global__ void __launch_bounds__(256) k_csf_force(Geom g, const float* __restrict__ F,
                                                   const float* __restrict__ kap, float* __restrict__ us,
                                                   float* __restrict__ vs, float* __restrict__ ws) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const int id = gidx(g, i, j, k);
    const float Fc = F[id], kc = kap[id];
    if (i >= 2) us[id] = us[id] + g.dt * csf_accel(g, F[id - 1], Fc, kap[id - 1], kc, g.dxi);
    if (j >= 2) vs[id] = vs[id] + g.dt * csf_accel(g, F[id - g.px], Fc, kap[id - g.px], kc, g.dyi);
    if (k >= 2) ws[id] = ws[id] + g.dt * csf_accel(g, F[id - g.plane], Fc, kap[id - g.plane], kc, g.dzi);
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
                                             float* __restrict__ rhs, int kchunk) {
    const Column col(g, 1, 1, kchunk);
    if (col.i > g.nx || col.j > g.ny || col.k0 > g.nz) return;
    int id = gidx(g, col.i, col.j, col.k0);
    float wsc = __ldg(ws + id);
    const float rdt = __frcp_rn(g.dt);
    // (unrolled so that the loads of several planes are in flight together)
#pragma unroll 4
    for (int k = col.k0; k <= col.k1; ++k, id += g.plane) {
        const float wsp = __ldg(ws + id + g.plane);
        const float rho = rho_of(g, __ldg(F + id));
        rhs[id] = div_rn_pre(rho, g.dt, rdt) *
                  ((__ldg(us + id + 1) - __ldg(us + id)) * g.dxi +
                   (__ldg(vs + id + g.px) - __ldg(vs + id)) * g.dyi +
                   (wsp - wsc) * g.dzi);
        wsc = wsp;
    }
}

// The same with four cells per thread: quads of a row as in k_correct4 (one
// aligned float4 word; quads of a plane numbered flat, one plane per
// blockIdx.y), every operand an aligned float4 load -- F, u*, v* of the row
// and of the row above, w* of the plane and of the plane above -- and the
// u* east of the quad's last cell from the next lane, or from memory at the
// end of a warp or of a row.  k_rhs's expression and operand order per cell.
__device__ __forceinline__ float4 ld4g(const float* __restrict__ a) {
    return __ldg(reinterpret_cast<const float4*>(a));
}
__device__ __forceinline__ float el4(const float4& v, int e) {
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

__global__ void __launch_bounds__(256) k_rhs4(Geom g, const float* __restrict__ F, const float* __restrict__ us,
                                              const float* __restrict__ vs, const float* __restrict__ ws,
                                              float* __restrict__ rhs) {
    const int nquad = g.nx / 4 + 1;  // quads covering columns 0 .. nx
    const int total = nquad * g.ny;
    const int qt = blockIdx.x * blockDim.x + threadIdx.x;
    const bool qa = qt < total;
    const int q = qa ? qt : total - 1;  // lanes past the end shadow the last quad
    const int jr = q / nquad, m = q - jr * nquad;
    const int j = jr + 1, k = blockIdx.y + 1, i0 = 4 * m;
    const int lane = threadIdx.x & 31;
    const bool lde = lane == 31 || m == nquad - 1;  // u* east of the quad from memory
    const int id = gidx(g, i0, j, k);  // a multiple of 4
    const float4 f4 = ld4g(F + id), u4 = ld4g(us + id), v4 = ld4g(vs + id), vn4 = ld4g(vs + id + g.px);
    const float4 w4 = ld4g(ws + id), wn4 = ld4g(ws + id + g.plane);
    const float ue_m = lde ? __ldg(us + id + 4) : 0.0f;
    float ue = __shfl_down_sync(0xffffffffu, u4.x, 1);
    if (lde) ue = ue_m;
    if (!qa) return;
    const float rdt = __frcp_rn(g.dt);
    float r[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float rho = rho_of(g, el4(f4, e));
        const float uip = e == 3 ? ue : el4(u4, e + 1);
        r[e] = div_rn_pre(rho, g.dt, rdt) * ((uip - el4(u4, e)) * g.dxi + (el4(vn4, e) - el4(v4, e)) * g.dyi +
                                             (el4(wn4, e) - el4(w4, e)) * g.dzi);
    }
    if (i0 >= 1 && i0 + 3 <= g.nx) {
        *reinterpret_cast<float4*>(rhs + id) = make_float4(r[0], r[1], r[2], r[3]);
        return;
    }
#pragma unroll
    for (int e = 0; e < 4; ++e)
        if (i0 + e >= 1 && i0 + e <= g.nx) rhs[id + e] = r[e];
}

// ---------------------------------------------------------------------------
// Velocity correction fused with the free-slip boundary conditions.
// update_{u,v,w}_kernel (voftrial1.cu:441-493) followed by apply_bc_velocity
// (voftrial1.cu:1107-1120, kernels :959-1051).  The three BC launches (j,
// then i, then k) compose to a closed form over the (nx+2)(ny+2)(nz+2) box,
// with c* an index clamped to the interior range and u_new the corrected
// face velocity:
//   u(i,j,k) = 0 for i == 1 or i == nx+1,  u_new(i, cj, ck) for 2 <= i <= nx,
//              u(0, cj, ck) (never updated) for i == 0
//   v(i,j,k) = 0 for j == 1 or j == ny+1,  v_new(ci, j, ck) for 2 <= j <= ny,
//              v(ci, 0, ck) for j == 0
//   w(i,j,k) = 0 for k == 1 or k == nz+1,  w_new(ci, cj, k) for 2 <= k <= nz,
//              w(ci, cj, 0) for k == 0
// The thread of interior cell (i,j,k) writes every box entry whose clamped
// source is its own, so each entry is written once and no thread reads an
// entry another thread writes.
//
// dt / r: faces between two pure cells have r in {rho_g, rho_l, (rho_g +
// rho_l)/2} (Geom::rpair); their IEEE quotients are formed once per context
// (Geom::qpair) and reused when r matches bit for bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float dt_over(const Geom& g, float r) {
    if (r == g.rpair[0]) return g.qpair[0];
    if (r == g.rpair[1]) return g.qpair[1];
    if (r == g.rpair[2]) return g.qpair[2];
    return g.dt / r;
}

__global__ void k_density_pairs(Geom g, float* out) {
    const float rg = rho_of(g, 0.0f), rl = rho_of(g, 1.0f);
    const float r0 = 0.5f * (rg + rg), r1 = 0.5f * (rl + rl), r2 = 0.5f * (rg + rl);
    out[0] = r0;
    out[1] = r1;
    out[2] = r2;
    out[3] = g.dt / r0;
    out[4] = g.dt / r1;
    out[5] = g.dt / r2;
}

struct EdgeDims {
    int nx, ny, nz, px, plane;
    __device__ int at(int i, int j, int k) const { return k * plane + j * px + i; }
};

// The boundary copies of a cell on the domain's edge.
__device__ __forceinline__ void store_edge_body(EdgeDims g, float* __restrict__ u, float* __restrict__ v,
                                                float* __restrict__ w, int i, int j, int k, float un, float vn,
                                                float wn) {
    int mi[3], mj[3], mk[3];
    const int nmi = mirrors(i, g.nx, mi), nmj = mirrors(j, g.ny, mj), nmk = mirrors(k, g.nz, mk);
    for (int b = 0; b < nmk; ++b)
        for (int a = 0; a < nmj; ++a) u[g.at(i, mj[a], mk[b])] = un;
    for (int b = 0; b < nmk; ++b)
        for (int a = 0; a < nmi; ++a) v[g.at(mi[a], j, mk[b])] = vn;
    for (int b = 0; b < nmj; ++b)
        for (int a = 0; a < nmi; ++a) w[g.at(mi[a], mj[b], k)] = wn;
    // far walls and the never-updated first planes
    if (i == g.nx)
        for (int b = 0; b < nmk; ++b)
            for (int a = 0; a < nmj; ++a) u[g.at(g.nx + 1, mj[a], mk[b])] = 0.0f;
    if (j == g.ny)
        for (int b = 0; b < nmk; ++b)
            for (int a = 0; a < nmi; ++a) v[g.at(mi[a], g.ny + 1, mk[b])] = 0.0f;
    if (k == g.nz)
        for (int b = 0; b < nmj; ++b)
            for (int a = 0; a < nmi; ++a) w[g.at(mi[a], mj[b], g.nz + 1)] = 0.0f;
    if (i == 1 && (nmj > 1 || nmk > 1)) {
        const float s0 = u[g.at(0, j, k)];
        for (int b = 0; b < nmk; ++b)
            for (int a = 0; a < nmj; ++a)
                if (a || b) u[g.at(0, mj[a], mk[b])] = s0;
    }
    if (j == 1 && (nmi > 1 || nmk > 1)) {
        const float s0 = v[g.at(i, 0, k)];
        for (int b = 0; b < nmk; ++b)
            for (int a = 0; a < nmi; ++a)
                if (a || b) v[g.at(mi[a], 0, mk[b])] = s0;
    }
    if (k == 1 && (nmi > 1 || nmj > 1)) {
        const float s0 = w[g.at(i, j, 0)];
        for (int b = 0; b < nmj; ++b)
            for (int a = 0; a < nmi; ++a)
                if (a || b) w[g.at(mi[a], mj[b], 0)] = s0;
    }
}

// The same out of line, for kernels that must not hold its registers.
static __device__ __noinline__ void store_edge(EdgeDims g, float* __restrict__ u, float* __restrict__ v,
                                               float* __restrict__ w, int i, int j, int k, float un, float vn,
                                               float wn) {
    store_edge_body(g, u, v, w, i, j, k, un, vn, wn);
}

// Writes the corrected face velocities of cell (i, j, k) and, on the domain
// edges, the boundary copies of apply_bc_velocity (voftrial1.cu:959-1051,
// 1107-1120) in closed form.  OUTLINE: the edge copies through a call.
template <bool OUTLINE>
__device__ __forceinline__ void store_corrected(const Geom& g, float* __restrict__ u, float* __restrict__ v,
                                                float* __restrict__ w, int i, int j, int k, int id, float un,
                                                float vn, float wn) {
    const bool edge_i = (i == 1 || i == g.nx), edge_j = (j == 1 || j == g.ny), edge_k = (k == 1 || k == g.nz);
    if (!(edge_i || edge_j || edge_k)) {  // bulk: one write per component
        u[id] = un;
        v[id] = vn;
        w[id] = wn;
        return;
    }
    const EdgeDims d{g.nx, g.ny, g.nz, g.px, g.plane};
    if (OUTLINE)
        store_edge(d, u, v, w, i, j, k, un, vn, wn);
    else
        store_edge_body(d, u, v, w, i, j, k, un, vn, wn);
}

__global__ void __launch_bounds__(256) k_correct(Geom g,
                                                 const float* __restrict__ F,
                                                 const float* __restrict__ us,
                                                 const float* __restrict__ vs,
                                                 const float* __restrict__ ws,
                                                 const float* __restrict__ p,
                                                 float* __restrict__ u, float* __restrict__ v,
                                                 float* __restrict__ w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const int sy = g.px, sz = g.plane;
    const int id = gidx(g, i, j, k);
    const float rho_c = rho_of(g, __ldg(F + id));
    const float p_c = __ldg(p + id);
    float un = 0.0f, vn = 0.0f, wn = 0.0f;  // wall faces (i, j or k == 1) are 0
    if (i >= 2) {
        const float r = 0.5f * (rho_c + rho_of(g, __ldg(F + id - 1)));
        un = __ldg(us + id) - dt_over(g, r) * (p_c - __ldg(p + id - 1)) * g.dxi;
    }
    if (j >= 2) {
        const float r = 0.5f * (rho_c + rho_of(g, __ldg(F + id - sy)));
        vn = __ldg(vs + id) - dt_over(g, r) * (p_c - __ldg(p + id - sy)) * g.dyi;
    }
    if (k >= 2) {
        const float r = 0.5f * (rho_c + rho_of(g, __ldg(F + id - sz)));
        wn = __ldg(ws + id) - dt_over(g, r) * (p_c - __ldg(p + id - sz)) * g.dzi;
    }
    store_corrected<false>(g, u, v, w, i, j, k, id, un, vn, wn);
}

// The correction with four cells per thread: a quad i = 4m .. 4m+3 of a row
// (one aligned float4 word of the padded layout; px is a multiple of 32), the
// quads of all rows of a plane numbered flat so that 32 consecutive quads
// make a warp across row ends, one plane per blockIdx.y.  Every operand is an
// aligned float4 load (the cell, its y-1 and its z-1 neighbours of F and p;
// u*, v*, w*); the x-1 neighbour of the quad's first cell comes from the
// lane before (its last cell's density and pressure), or from memory at the
// start of a warp.  Each face keeps k_correct's expression and operand order
// (same bits).  Quads without an edge cell store float4 words; the others go
// through store_corrected cell by cell.
__global__ void __launch_bounds__(256, 4) k_correct4(Geom g, const float* __restrict__ F,
                                                  const float* __restrict__ us, const float* __restrict__ vs,
                                                  const float* __restrict__ ws, const float* __restrict__ p,
                                                  float* __restrict__ u, float* __restrict__ v,
                                                  float* __restrict__ w) {
    const int nquad = g.nx / 4 + 1;  // quads covering columns 0 .. nx
    const int total = nquad * g.ny;
    const int qt = blockIdx.x * blockDim.x + threadIdx.x;
    const bool qa = qt < total;
    const int q = qa ? qt : total - 1;  // lanes past the end shadow the last quad
    const int jr = q / nquad, m = q - jr * nquad;
    const int j = jr + 1, k = blockIdx.y + 1, i0 = 4 * m;
    const int lane = threadIdx.x & 31;
    const bool ldw = lane == 0 && m > 0;  // the x-1 neighbour from memory
    const int sy = g.px, sz = g.plane;
    const int id = gidx(g, i0, j, k);  // a multiple of 4
    const float4 fc = ld4g(F + id), fs = ld4g(F + id - sy), fb = ld4g(F + id - sz);
    const float4 pc = ld4g(p + id), ps = ld4g(p + id - sy), pb = ld4g(p + id - sz);
    const float4 u4 = ld4g(us + id), v4 = ld4g(vs + id), w4 = ld4g(ws + id);
    const float fl = ldw ? __ldg(F + id - 1) : 0.0f, pl = ldw ? __ldg(p + id - 1) : 0.0f;
    float rc[4] = {rho_of(g, fc.x), rho_of(g, fc.y), rho_of(g, fc.z), rho_of(g, fc.w)};
    float rl = __shfl_up_sync(0xffffffffu, rc[3], 1), pw = __shfl_up_sync(0xffffffffu, pc.w, 1);
    if (ldw) {
        rl = rho_of(g, fl);
        pw = pl;
    }
    float un[4], vn[4], wn[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int i = i0 + e;
        const float rho_c = rc[e], p_c = el4(pc, e);
        un[e] = 0.0f;  // wall faces (i, j or k == 1) are 0
        vn[e] = 0.0f;
        wn[e] = 0.0f;
        if (i >= 2) {
            const float r = 0.5f * (rho_c + (e == 0 ? rl : rc[e - 1]));
            un[e] = el4(u4, e) - dt_over(g, r) * (p_c - (e == 0 ? pw : el4(pc, e - 1))) * g.dxi;
        }
        if (j >= 2) {
            const float r = 0.5f * (rho_c + rho_of(g, el4(fs, e)));
            vn[e] = el4(v4, e) - dt_over(g, r) * (p_c - el4(ps, e)) * g.dyi;
        }
        if (k >= 2) {
            const float r = 0.5f * (rho_c + rho_of(g, el4(fb, e)));
            wn[e] = el4(w4, e) - dt_over(g, r) * (p_c - el4(pb, e)) * g.dzi;
        }
    }
    if (!qa) return;
    const bool bulk = i0 >= 2 && i0 + 3 <= g.nx - 1 && j != 1 && j != g.ny && k != 1 && k != g.nz;
    if (bulk) {
        *reinterpret_cast<float4*>(u + id) = make_float4(un[0], un[1], un[2], un[3]);
        *reinterpret_cast<float4*>(v + id) = make_float4(vn[0], vn[1], vn[2], vn[3]);
        *reinterpret_cast<float4*>(w + id) = make_float4(wn[0], wn[1], wn[2], wn[3]);
        return;
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int i = i0 + e;
        if (i >= 1 && i <= g.nx) store_corrected<true>(g, u, v, w, i, j, k, id + e, un[e], vn[e], wn[e]);
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
cudaError_t plain_configure(int max_line) {
    (void)max_line;
    cudaError_t e = fct_configure();
    return e == cudaSuccess ? jacobi_tb_configure() : e;
}

cudaError_t plain_density_pairs(Geom* g) {
    float* d = nullptr;
    float h[6];
    cudaError_t e = cudaMalloc(&d, sizeof(h));
    if (e != cudaSuccess) return e;
    k_density_pairs<<<1, 1>>>(*g, d);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return e;
    for (int q = 0; q < 3; ++q) {
        g->rpair[q] = h[q];
        g->qpair[q] = h[3 + q];
    }
    return cudaSuccess;
}

cudaError_t plain_density_pairs_on(Geom* g, float* dev6, cudaStream_t s) {
    float h[6];
    k_density_pairs<<<1, 1, 0, s>>>(*g, dev6);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, dev6, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    for (int q = 0; q < 3; ++q) {
        g->rpair[q] = h[q];
        g->qpair[q] = h[3 + q];
    }
    return cudaSuccess;
}

bool plain_supported(const Geom& g) {
    return fct_smem_bytes(0, g.nx) <= fct_smem_limit() && fct_smem_bytes(1, g.ny) <= fct_smem_limit() &&
           fct_smem_bytes(2, g.nz) <= fct_smem_limit();
}

// Sweeps fused per Jacobi launch (1 .. JACOBI_TB_MAX).
#ifndef VOF_JACOBI_T
#define VOF_JACOBI_T 2
#endif
constexpr int JACOBI_T = VOF_JACOBI_T;
static_assert(JACOBI_T >= 1 && JACOBI_T <= JACOBI_TB_MAX, "VOF_JACOBI_T out of range");

// Launches for `iters` sweeps: ceil(iters / JACOBI_T), except that a single
// blocked launch cannot end in the buffer it reads, so iters == JACOBI_T
// (even) runs as single sweeps.
// Jacobi kernels.  One sweep per launch: two cells per thread with the
// plane cases peeled out of the z march (k_jacobi_peel, the default), the
// same without the peeling (k_jacobi_pairs), with its own column's loads
// copied several planes ahead (k_jacobi_ring), fed by bulk copies of whole
// rows (k_jacobi_bulk), with four cells per thread (k_jacobi_quad), with one
// cell per thread (k_jacobi_col), or through TMA tiles (k_jacobi_tb, one
// sweep: tb1).  Several sweeps per launch: two cells per thread, two sweeps
// (k_jacobi_pairs2; an odd count starts with one single sweep), or JACOBI_T
// temporally blocked sweeps through TMA (k_jacobi_tb).
// VOF_JACOBI=peel|pairs|ring|bulk|quad|col|tb1|pairs2|tb forces one.  All
// give the same bits.
enum { JACOBI_PAIRS = 0, JACOBI_COL = 1, JACOBI_TB = 2, JACOBI_PAIRS2 = 3, JACOBI_RING = 4, JACOBI_PEEL = 5, JACOBI_TB1 = 6, JACOBI_BULK = 7, JACOBI_QUAD = 8 };
static int jacobi_kind(const Geom& g) {
    static int forced = -2;
    if (forced == -2) {
        const char* v = getenv("VOF_JACOBI");
        forced = -1;
        if (v && !strcmp(v, "pairs")) forced = JACOBI_PAIRS;
        if (v && !strcmp(v, "col")) forced = JACOBI_COL;
        if (v && !strcmp(v, "tb")) forced = JACOBI_TB;
        if (v && !strcmp(v, "pairs2")) forced = JACOBI_PAIRS2;
        if (v && !strcmp(v, "ring")) forced = JACOBI_RING;
        if (v && !strcmp(v, "peel")) forced = JACOBI_PEEL;
        if (v && !strcmp(v, "tb1")) forced = JACOBI_TB1;
        if (v && !strcmp(v, "bulk")) forced = JACOBI_BULK;
        if (v && !strcmp(v, "quad")) forced = JACOBI_QUAD;
    }
    const int k = forced >= 0 ? forced : JACOBI_PEEL;
    if (k == JACOBI_BULK && !jacobi_bulk_supported(g)) return JACOBI_PAIRS;
    return (k == JACOBI_PAIRS2 && !jacobi_pairs2_supported(g)) ? JACOBI_PAIRS : k;
}
// The peeled kernel marches z downwards on every second sweep when the
// three buffers the sweeps touch (two pressures and rhs) are at most 1.25x
// the L2: a sweep then starts on the planes the previous one touched last,
// which are still in L2, instead of on the ones touched first, which a
// cyclic march has evicted.  Measured on a B200: 200^3 (110 MB) 4 % faster
// sweeps, 128^3 (all in L2) unchanged, 256^3 (230 MB) 1 % slower.
// VOF_JACOBI_ALT=0 / 1 forces it off / on.
static bool jacobi_alternate(const Geom& g) {
    static int forced = -2;
    static long long l2 = 0;
    if (forced == -2) {
        const char* v = getenv("VOF_JACOBI_ALT");
        forced = v ? (atoi(v) != 0 ? 1 : 0) : -1;
        int dev = 0, b = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&b, cudaDevAttrL2CacheSize, dev) == cudaSuccess)
            l2 = b;
    }
    if (forced >= 0) return forced == 1;
    const long long bytes = 3LL * g.plane * (g.nz + 2) * (long long)sizeof(float);
    return l2 > 0 && 4 * bytes <= 5 * l2;
}

static bool jacobi_streaming(const Geom& g) {
    const int k = jacobi_kind(g);
    return k == JACOBI_PAIRS || k == JACOBI_COL || k == JACOBI_RING || k == JACOBI_PEEL || k == JACOBI_BULK ||
           k == JACOBI_QUAD;
}
static int jacobi_per_launch(const Geom& g) {
    const int k = jacobi_kind(g);
    return k == JACOBI_PAIRS2 ? 2 : k == JACOBI_TB1 ? 1 : JACOBI_T;
}

static int jacobi_launches(const Geom& g, int iters) {
    if (jacobi_streaming(g)) return iters;
    const int T = jacobi_per_launch(g);
    const int L = (iters + T - 1) / T;
    return (L == 1 && iters % 2 == 0) ? iters : L;
}

// Buffer sequence for L blocked launches taking the pressure from physical
// buffer `src` to `dst` (0/1: the two buffers the reference ping-pongs; 2: a
// scratch buffer), consecutive buffers distinct.  Returns false when no such
// sequence exists (L == 1 with src == dst).
static bool plan_buffers(int src, int dst, int L, int* seq) {
    if (L == 0) return src == dst;
    if (L == 1 && src == dst) return false;
    seq[0] = src;
    seq[L] = dst;
    for (int q = L - 1; q >= 1; --q) {
        int c = 2;
        if (c == seq[q + 1]) c = (seq[q + 1] == 0) ? 1 : 0;
        if (q == 1 && c == src) {
            for (int t = 0; t < 3; ++t)
                if (t != src && t != seq[2]) c = t;
        }
        seq[q] = c;
    }
    return true;
}

int plain_kernels_per_step(const Geom& g, int jacobi_iters) {
    return 1 + (g.csf ? 3 : 0) + 1 + jacobi_launches(g, jacobi_iters) + 1 + 3;
}

// Column-marching launch shape: 32 x 8 columns per block, z split into
// chunks of about 16 planes (long enough to reuse the k-window, short enough
// for a few waves of blocks per SM).  On small grids the chunks shrink (down
// to one plane) until the launch has about 600 blocks: a launch of a few
// blocks marching 16 planes each is bound by the latency of its march.
static void column_launch(const Geom& g, dim3& grid, int& kchunk) {
    const int bx = (g.nx + TX - 1) / TX, by = (g.ny + TY - 1) / TY;
    const int target = (int)(((long long)g.nz * bx * by) / 600);
    const int len = target < 1 ? 1 : (target > 16 ? 16 : target);
    const int nch = (g.nz + len - 1) / len;
    kchunk = (g.nz + nch - 1) / nch;
    grid = dim3(bx, by, (g.nz + kchunk - 1) / kchunk);
}

// ev (optional, PLAIN_PHASES+1 events): ev[0] before the step, ev[q+1]
// after phase q (predict, rhs, pressure, correct, sweep 1, sweep 2, sweep 3).
static inline cudaError_t mark(cudaEvent_t* ev, int q, cudaStream_t s) {
    return ev ? cudaEventRecord(ev[q], s) : cudaSuccess;
}

// Four-cell kernels (k_rhs4, k_correct4) when their launch has at least
// about 7 blocks per SM of a B200 (measured: faster from 128^3 up, slower at
// 32^3 and 64^3, where the one-cell kernels' four times as many threads
// fill the GPU better).  VOF_RHS / VOF_CORRECT = 1 or 4 force either.
static bool quads_fill(const Geom& g) {
    const long long blocks = (long long)(((g.nx / 4 + 1) * g.ny + 255) / 256) * g.nz;
    return blocks >= 1024;
}
// SMs of the current device (queried once).
static int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
                                                      cudaSuccess)
            n = 148;
    }
    return n;
}

// 1: the one-cell kernel, 4: the four-cell kernel, else by size.
static int env_kernel(const char* name) {
    const char* v = getenv(name);
    return v ? atoi(v) : 0;
}

cudaError_t plain_front(const Geom& g, const PlainBuffers& b, cudaStream_t s, cudaEvent_t* ev) {
    const dim3 blk(TX, TY, 1);
    dim3 grid;
    int kchunk = 1;
    column_launch(g, grid, kchunk);
    cudaError_t e;
    if ((e = mark(ev, 0, s)) != cudaSuccess) return e;
    static int pforced = -1;  // VOF_PREDICT=1: k_predict (one cell per thread); else k_predict2
    if (pforced < 0) pforced = env_kernel("VOF_PREDICT");
    if (pforced == 1) {
        k_predict<<<grid, blk, 0, s>>>(g, b.F, b.u, b.v, b.w, b.us, b.vs, b.ws, kchunk);
    } else {
        const int bx = ((g.nx / 2 + 1) * g.ny + 255) / 256;
        const int kc = wave_kchunk(g.nz, bx, 4 * sm_count());
        k_predict2<<<dim3(bx, (g.nz + kc - 1) / kc), 256, 0, s>>>(g, b.F, b.u, b.v, b.w, b.us, b.vs, b.ws, kc);
    }
    if (g.csf && b.csf[0]) {  // surface tension (extension): normals, curvature, face accelerations
        const dim3 cb(32, 4, 2);
        const dim3 cg((g.nx + 31) / 32, (g.ny + 3) / 4, (g.nz + 1) / 2);
        k_csf_normal<<<cg, cb, 0, s>>>(g, b.F, b.csf[0], b.csf[1], b.csf[2]);
        k_csf_curv<<<cg, cb, 0, s>>>(g, b.csf[0], b.csf[1], b.csf[2], b.csf[3]);
        k_csf_force<<<cg, cb, 0, s>>>(g, b.F, b.csf[3], b.us, b.vs, b.ws);
    }
    if ((e = cudaGetLastError()) != cudaSuccess || (e = mark(ev, 1, s)) != cudaSuccess) return e;
    static int forced = -1;  // VOF_RHS=1: k_rhs (one cell per thread, z march), 4: k_rhs4
    if (forced < 0) forced = env_kernel("VOF_RHS");
    if (forced == 1 || (forced != 4 && !quads_fill(g))) {
        k_rhs<<<grid, blk, 0, s>>>(g, b.F, b.us, b.vs, b.ws, b.rhs, kchunk);
    } else {
        const int total = (g.nx / 4 + 1) * g.ny;
        k_rhs4<<<dim3((total + 255) / 256, g.nz), 256, 0, s>>>(g, b.F, b.us, b.vs, b.ws, b.rhs);
    }
    if ((e = cudaGetLastError()) != cudaSuccess || (e = mark(ev, 2, s)) != cudaSuccess) return e;
    return cudaSuccess;
}

// The correction: k_correct4 (four cells per thread) on large grids, else
// k_correct (one cell per thread).  Both give the same bits.
cudaError_t plain_correct(const Geom& g, const PlainBuffers& b, const float* p, cudaStream_t s) {
    static int forced = -1;
    if (forced < 0) forced = env_kernel("VOF_CORRECT");
    if (forced == 1 || (forced != 4 && !quads_fill(g))) {
        const dim3 cb(32, 4, 2);
        const dim3 cg((g.nx + 31) / 32, (g.ny + 3) / 4, (g.nz + 1) / 2);
        k_correct<<<cg, cb, 0, s>>>(g, b.F, b.us, b.vs, b.ws, p, b.u, b.v, b.w);
    } else {
        const int total = (g.nx / 4 + 1) * g.ny;
        k_correct4<<<dim3((total + 255) / 256, g.nz), 256, 0, s>>>(g, b.F, b.us, b.vs, b.ws, p, b.u, b.v, b.w);
    }
    return cudaGetLastError();
}

cudaError_t plain_back(const Geom& g, const PlainBuffers& b, int istep, const float* p, cudaStream_t s,
                       cudaEvent_t* ev) {
    cudaError_t e;
    if ((e = mark(ev, 3, s)) != cudaSuccess) return e;
    if ((e = plain_correct(g, b, p, s)) != cudaSuccess || (e = mark(ev, 4, s)) != cudaSuccess) return e;

    // Sweep order by istep % 3 (voftrial1.cu:1384-1396).  The sweeps run out
    // of place, F -> s1 -> s2 -> F, through the two pressure buffers that do
    // not hold the pressure: the next step's solve writes their interiors
    // before it reads them, and their ghost cells (never written by a sweep or
    // a Jacobi launch) hold finite values, which a sweep reads only through
    // the zero velocity of a wall face.
    const int r = ((istep % 3) + 3) % 3;
    static const int order[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
    float* s1 = (p == b.p0) ? b.p1 : b.p0;
    float* s2 = b.p2;
    const bool oop = s1 && s2 && p != b.p2;
    const float* src[3] = {b.F, s1, s2};
    float* dst[3] = {s1, s2, b.F};
    for (int q = 0; q < 3; ++q) {
        const int axis = order[r][q];
        const float* vel = axis == 0 ? b.u : (axis == 1 ? b.v : b.w);
        e = oop ? fct_launch_to(g, axis, q == 2, src[q], dst[q], vel, s) : fct_launch(g, axis, q == 2, b.F, vel, s);
        if (e != cudaSuccess || (e = mark(ev, 5 + q, s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t plain_pressure(const Geom& g, const PlainBuffers& b, int jacobi_iters, int* p_parity, cudaStream_t s) {
    cudaError_t e;

    // Jacobi (voftrial1.cu:1371-1375): one streaming sweep per launch on
    // small grids, else JACOBI_T blocked sweeps per launch.  The
    // reference ping-pongs p <-> pt once per sweep, so after N sweeps its
    // pressure sits in the buffer it started in when N is even and in the
    // other one when N is odd; the launches route through the scratch
    // buffer so the result lands in that same buffer (which keeps the
    // reference's ghost entries in a download).
    float* pbuf[3] = {b.p0, b.p1, b.p2};
    const int src = *p_parity, dst = src ^ (jacobi_iters & 1);
    const int T = jacobi_per_launch(g);
    const int L = (jacobi_iters + T - 1) / T;
    int seq[64];
    if (jacobi_kind(g) == JACOBI_PAIRS2 && L <= 62 && plan_buffers(src, dst, L, seq)) {
        // an odd count starts with one single sweep
        for (int q = 0; q < L; ++q) {
            const bool single = q == 0 && (jacobi_iters & 1);
            e = single ? jacobi_pairs_launch(g, pbuf[seq[q]], b.rhs, pbuf[seq[q + 1]], s)
                       : jacobi_pairs2_launch(g, pbuf[seq[q]], b.rhs, pbuf[seq[q + 1]], s);
            if (e != cudaSuccess) return e;
        }
    } else if (jacobi_streaming(g) || jacobi_kind(g) == JACOBI_PAIRS2) {
        int cur = src;
        const int kind = jacobi_kind(g);
        const bool alt = kind == JACOBI_PEEL && jacobi_alternate(g);
        for (int it = 0; it < jacobi_iters; ++it) {
            e = kind == JACOBI_COL    ? jacobi_col_launch(g, pbuf[cur], b.rhs, pbuf[cur ^ 1], s)
                : kind == JACOBI_RING ? jacobi_ring_launch(g, pbuf[cur], b.rhs, pbuf[cur ^ 1], s)
                : kind == JACOBI_PEEL ? jacobi_peel_launch(g, pbuf[cur], b.rhs, pbuf[cur ^ 1], s,
                                                           alt && (it & 1))
                : kind == JACOBI_BULK ? jacobi_bulk_launch(g, pbuf[cur], b.rhs, pbuf[cur ^ 1], b.status, s)
                : kind == JACOBI_QUAD ? jacobi_quad_launch(g, pbuf[cur], b.rhs, pbuf[cur ^ 1], s)
                                      : jacobi_pairs_launch(g, pbuf[cur], b.rhs, pbuf[cur ^ 1], s);
            if (e != cudaSuccess) return e;
            cur ^= 1;
        }
    } else if (L > 62 || !plan_buffers(src, dst, L, seq)) {
        // fall back to one sweep per launch: a plain ping-pong always works
        int cur = src;
        for (int it = 0; it < jacobi_iters; ++it) {
            if ((e = jacobi_tb_launch(g, 1, b.maps[cur], b.maps[3], pbuf[cur ^ 1], b.status, s)) != cudaSuccess)
                return e;
            cur ^= 1;
        }
    } else {
        const int T1 = jacobi_per_launch(g);
        for (int q = 0; q < L; ++q) {
            const int T = (q == 0 && jacobi_iters % T1) ? jacobi_iters % T1 : T1;
            if ((e = jacobi_tb_launch(g, T, b.maps[seq[q]], b.maps[3], pbuf[seq[q + 1]], b.status, s)) !=
                cudaSuccess)
                return e;
        }
    }
    *p_parity = dst;
    return cudaSuccess;
}

cudaError_t plain_step(const Geom& g, const PlainBuffers& b, int istep, int jacobi_iters,
                       int* p_parity, cudaStream_t s, cudaEvent_t* ev) {
    cudaError_t e = plain_front(g, b, s, ev);
    if (e != cudaSuccess) return e;
    if ((e = plain_pressure(g, b, jacobi_iters, p_parity, s)) != cudaSuccess) return e;
    float* pbuf[3] = {b.p0, b.p1, b.p2};
    return plain_back(g, b, istep, pbuf[*p_parity], s, ev);
}

int plain_phase_launches(const Geom& g, int phase, int jacobi_iters) {
    if (phase == PHASE_JACOBI) return jacobi_launches(g, jacobi_iters);
    return (phase == PHASE_PREDICT && g.csf) ? 4 : 1;
}

}  // namespace vof
