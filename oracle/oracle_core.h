// oracle_core.h -- the CPU restatement of the voftrial1.cu time step, shared
// by vof_oracle.cpp (the forward oracle) and vof_adjoint.cpp (its adjoint).
//
// TEST INFRASTRUCTURE ONLY: included by the oracle sources under oracle/, never by
// the product.
//
// It follows the reference kernel by kernel, with all twenty DeviceFields
// buffers (voftrial1.cu:1176-1198) in the reference layout, zero-filled at the
// start of a run like alloc_field (voftrial1.cu:1200-1203), and in the launch
// order of the time loop (voftrial1.cu:1361-1401).  It is templated on the
// scalar type:
//   float  -- built with -ffp-contract=off: IEEE single precision with no
//             fused multiply-add, i.e. the reference's arithmetic as written.
//             The reference's kernels compiled with nvcc -fmad=false produce
//             the same bits (pinned by the fixtures in tests/golden).
//   double -- the FP64 oracle: the same expressions in double precision
//             (median3 then quantises at 2^-52 instead of 2^-23).
// and on a switch policy (Plain: the arithmetic as written; Taped: record or
// replay every non-smooth choice).
// Loops over k are split across OpenMP threads; inside a k-plane the order is
// sequential, so the reference's benign duplicate face writes
// (voftrial1.cu:572-575) store the same value twice, as on the GPU.  A Taped
// oracle runs with one thread, so its tape has one fixed order.
#pragma once
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "../include/vof.h"

namespace vofo {

template <typename T>
struct Prm {
    int nx, ny, nz;
    T Lx, Ly, Lz, rho_l, rho_g, nu_l, nu_g, gx, gy, gz, dt;
    T dx, dy, dz, dxi, dyi, dzi;
    int jacobi_iters;
};

// float: the caller's float parameters as they are (they come from
// vof_params_init/finalize, the reference's own expressions).
inline Prm<float> make_prm(const vof_params* p, float) {
    Prm<float> q;
    q.nx = p->nx; q.ny = p->ny; q.nz = p->nz;
    q.Lx = p->Lx; q.Ly = p->Ly; q.Lz = p->Lz;
    q.rho_l = p->rho_l; q.rho_g = p->rho_g; q.nu_l = p->nu_l; q.nu_g = p->nu_g;
    q.gx = p->gx; q.gy = p->gy; q.gz = p->gz; q.dt = p->dt;
    q.dx = p->dx; q.dy = p->dy; q.dz = p->dz;
    q.dxi = p->dxi; q.dyi = p->dyi; q.dzi = p->dzi;
    q.jacobi_iters = p->jacobi_iters;
    return q;
}

// double: the primary float constants promoted, the derived lengths formed in
// double with the same expressions as voftrial1.cu:1285-1290.
inline Prm<double> make_prm(const vof_params* p, double) {
    Prm<double> q;
    q.nx = p->nx; q.ny = p->ny; q.nz = p->nz;
    q.Lx = p->Lx; q.Ly = p->Ly; q.Lz = p->Lz;
    q.rho_l = p->rho_l; q.rho_g = p->rho_g; q.nu_l = p->nu_l; q.nu_g = p->nu_g;
    q.gx = p->gx; q.gy = p->gy; q.gz = p->gz; q.dt = p->dt;
    q.dx = q.Lx / q.nx; q.dy = q.Ly / q.ny; q.dz = q.Lz / q.nz;
    q.dxi = 1.0 / q.dx; q.dyi = 1.0 / q.dy; q.dzi = 1.0 / q.dz;
    q.jacobi_iters = p->jacobi_iters;
    return q;
}

// voftrial1.cu:52-60
template <typename T>
inline T median3(T a, T b, T c) {
    const T mx = std::fmax(std::fmax(a, b), c);
    const T mn = std::fmin(std::fmin(a, b), c);
    return a + b + c - mx - mn;
}
template <typename T>
inline T clamp01(T v) { return median3<T>(T(0), T(1), v); }

// Switch policies of Oracle.  Every non-smooth choice of the step goes through
// one of: br(c) (a branch condition), mx(a, b) / mn(a, b) (fmax / fmin, the
// first argument winning a tie).  Plain evaluates them as written (the
// reference's arithmetic); Taped records the outcomes of a base run and can
// replay them, which freezes the switches (the piecewise-smooth map of the
// base point) for finite differences and defines the derivative the adjoint
// takes at a tie.
struct Plain {
    static inline bool br(bool c) { return c; }
    template <typename T>
    static inline T mx(T a, T b) { return std::fmax(a, b); }
    template <typename T>
    static inline T mn(T a, T b) { return std::fmin(a, b); }
};

struct Taped {
    std::vector<uint8_t>* bits = nullptr;  // the tape
    bool replay = false;
    size_t pos = 0;
    bool overrun = false;                  // replay ran past the tape
    inline bool take(bool c) {
        if (!replay) {
            bits->push_back((uint8_t)c);
            return c;
        }
        if (pos >= bits->size()) {
            overrun = true;
            return c;
        }
        return (*bits)[pos++] != 0;
    }
    inline bool br(bool c) { return take(c); }
    template <typename T>
    inline T mx(T a, T b) { return take(a >= b) ? a : b; }
    template <typename T>
    inline T mn(T a, T b) { return take(a <= b) ? a : b; }
};

template <typename T, typename SW = Plain>
struct Oracle {
    Prm<T> P;
    SW sw;
    int NX, NY, NZ;  // extents with ghosts
    size_t N;
    // DeviceFields (voftrial1.cu:1176-1198)
    std::vector<T> F, Ftd, ax, ay, az, cx, cy, cz, rp, rm, u, v, w, us, vs, ws, p, pt, rho, nu;
    int nthreads;

    explicit Oracle(const Prm<T>& prm, int nth) : P(prm), nthreads(nth) {
        NX = P.nx + 2; NY = P.ny + 2; NZ = P.nz + 2;
        N = (size_t)NX * NY * NZ;
        for (auto* f : {&F, &Ftd, &ax, &ay, &az, &cx, &cy, &cz, &rp, &rm, &u, &v, &w, &us, &vs, &ws, &p,
                        &pt, &rho, &nu})
            f->assign(N, T(0));
    }
    // idx3d, voftrial1.cu:66-70
    inline size_t id(int i, int j, int k) const { return ((size_t)k * NY + j) * NX + i; }

    // clamp01 through the switch policy: median3(0, 1, v) with
    // fmax(fmax(0,1), v) = mx(1, v) and fmin(fmin(0,1), v) = mn(0, v).
    inline T clamp01s(T v) {
        const T hi = sw.mx(T(1), v);
        const T lo = sw.mn(T(0), v);
        return T(0) + T(1) + v - hi - lo;
    }

    // cal_nu_rho_kernel, voftrial1.cu:95-104 (every cell, ghosts included)
    void cal_nu_rho() {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long long t = 0; t < (long long)N; ++t) {
            const T f = clamp01s(F[t]);
            rho[t] = P.rho_g * (T(1) - f) + P.rho_l * f;
            nu[t] = P.nu_l * f + P.nu_g * (T(1) - f);
        }
    }

    // advect_u_kernel, voftrial1.cu:230-285 (i in [imin+1, imax])
    void advect_u() {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 2; i <= P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    const T v_here = T(0.25) * (v[id(i - 1, j, k)] + v[id(i - 1, j + 1, k)] + v[id(i, j, k)] +
                                                v[id(i, j + 1, k)]);
                    const T w_here = T(0.25) * (w[id(i - 1, j, k)] + w[id(i - 1, j, k + 1)] + w[id(i, j, k)] +
                                                w[id(i, j, k + 1)]);
                    const T uc = u[c];
                    const T um = u[id(i - 1, j, k)], up = u[id(i + 1, j, k)];
                    const T ujm = u[id(i, j - 1, k)], ujp = u[id(i, j + 1, k)];
                    const T ukm = u[id(i, j, k - 1)], ukp = u[id(i, j, k + 1)];
                    const T dudx = sw.br(uc > T(0)) ? (uc - um) * P.dxi : (up - uc) * P.dxi;
                    const T dudy = sw.br(v_here > T(0)) ? (uc - ujm) * P.dyi : (ujp - uc) * P.dyi;
                    const T dudz = sw.br(w_here > T(0)) ? (uc - ukm) * P.dzi : (ukp - uc) * P.dzi;
                    const T visc = nu[c] * (um - T(2) * uc + up) * P.dxi * P.dxi +
                                   nu[c] * (ujm - T(2) * uc + ujp) * P.dyi * P.dyi +
                                   nu[c] * (ukm - T(2) * uc + ukp) * P.dzi * P.dzi;
                    const T adv = -uc * dudx - v_here * dudy - w_here * dudz;
                    us[c] = uc + P.dt * (visc + adv + P.gx);
                }
    }

    // advect_v_kernel, voftrial1.cu:287-342 (j in [jmin+1, jmax])
    void advect_v() {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 2; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    const T u_here = T(0.25) * (u[id(i, j - 1, k)] + u[id(i, j, k)] + u[id(i + 1, j - 1, k)] +
                                                u[id(i + 1, j, k)]);
                    const T w_here = T(0.25) * (w[id(i, j - 1, k + 1)] + w[id(i, j - 1, k)] + w[id(i, j, k)] +
                                                w[id(i, j, k + 1)]);
                    const T vc = v[c];
                    const T vim = v[id(i - 1, j, k)], vip = v[id(i + 1, j, k)];
                    const T vjm = v[id(i, j - 1, k)], vjp = v[id(i, j + 1, k)];
                    const T vkm = v[id(i, j, k - 1)], vkp = v[id(i, j, k + 1)];
                    const T dvdx = sw.br(u_here > T(0)) ? (vc - vim) * P.dxi : (vip - vc) * P.dxi;
                    const T dvdy = sw.br(vc > T(0)) ? (vc - vjm) * P.dyi : (vjp - vc) * P.dyi;
                    const T dvdz = sw.br(w_here > T(0)) ? (vc - vkm) * P.dzi : (vkp - vc) * P.dzi;
                    const T visc = nu[c] * (vim - T(2) * vc + vip) * P.dxi * P.dxi +
                                   nu[c] * (vjm - T(2) * vc + vjp) * P.dyi * P.dyi +
                                   nu[c] * (vkm - T(2) * vc + vkp) * P.dzi * P.dzi;
                    const T adv = -u_here * dvdx - vc * dvdy - w_here * dvdz;
                    vs[c] = vc + P.dt * (visc + adv + P.gy);
                }
    }

    // advect_w_kernel, voftrial1.cu:344-399 (k in [kmin+1, kmax])
    void advect_w() {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 2; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    const T u_here = T(0.25) * (u[id(i + 1, j, k - 1)] + u[id(i, j, k - 1)] + u[id(i + 1, j, k)] +
                                                u[id(i, j, k)]);
                    const T v_here = T(0.25) * (v[id(i, j + 1, k - 1)] + v[id(i, j, k - 1)] + v[id(i, j, k)] +
                                                v[id(i, j + 1, k)]);
                    const T wc = w[c];
                    const T wim = w[id(i - 1, j, k)], wip = w[id(i + 1, j, k)];
                    const T wjm = w[id(i, j - 1, k)], wjp = w[id(i, j + 1, k)];
                    const T wkm = w[id(i, j, k - 1)], wkp = w[id(i, j, k + 1)];
                    const T dwdx = sw.br(u_here > T(0)) ? (wc - wim) * P.dxi : (wip - wc) * P.dxi;
                    const T dwdy = sw.br(v_here > T(0)) ? (wc - wjm) * P.dyi : (wjp - wc) * P.dyi;
                    const T dwdz = sw.br(wc > T(0)) ? (wc - wkm) * P.dzi : (wkp - wc) * P.dzi;
                    const T visc = nu[c] * (wim - T(2) * wc + wip) * P.dxi * P.dxi +
                                   nu[c] * (wjm - T(2) * wc + wjp) * P.dyi * P.dyi +
                                   nu[c] * (wkm - T(2) * wc + wkp) * P.dzi * P.dzi;
                    const T adv = -u_here * dwdx - v_here * dwdy - wc * dwdz;
                    ws[c] = wc + P.dt * (visc + adv + P.gz);
                }
    }

    // rhs term of solve_p_jacobi_kernel, voftrial1.cu:418-422
    inline T rhs_at(int i, int j, int k) const {
        const size_t c = id(i, j, k);
        return rho[c] / P.dt *
               ((us[id(i + 1, j, k)] - us[c]) * P.dxi + (vs[id(i, j + 1, k)] - vs[c]) * P.dyi +
                (ws[id(i, j, k + 1)] - ws[c]) * P.dzi);
    }

    // solve_p_jacobi_kernel, voftrial1.cu:401-439: reads p, writes pt.
    void jacobi_sweep(const std::vector<T>& pin, std::vector<T>& pout) {
        const T cx = P.dxi * P.dxi, cyy = P.dyi * P.dyi, cz = P.dzi * P.dzi;
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) {
                    const T rhs = rhs_at(i, j, k);
                    const T ae = (i != P.nx) ? cx : T(0);
                    const T aw = (i != 1) ? cx : T(0);
                    const T an = (j != P.ny) ? cyy : T(0);
                    const T as = (j != 1) ? cyy : T(0);
                    const T af = (k != P.nz) ? cz : T(0);
                    const T ab = (k != 1) ? cz : T(0);
                    const T ap = -(ae + aw + an + as + af + ab);
                    pout[id(i, j, k)] = (rhs - ae * pin[id(i + 1, j, k)] - aw * pin[id(i - 1, j, k)] -
                                         an * pin[id(i, j + 1, k)] - as * pin[id(i, j - 1, k)] -
                                         af * pin[id(i, j, k + 1)] - ab * pin[id(i, j, k - 1)]) /
                                        ap;
                }
    }

    // update_{u,v,w}_kernel, voftrial1.cu:441-493
    void update_uvw() {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    if (i >= 2) {
                        const size_t m = id(i - 1, j, k);
                        const T r = T(0.5) * (rho[c] + rho[m]);
                        u[c] = us[c] - P.dt / r * (p[c] - p[m]) * P.dxi;
                    }
                    if (j >= 2) {
                        const size_t m = id(i, j - 1, k);
                        const T r = T(0.5) * (rho[c] + rho[m]);
                        v[c] = vs[c] - P.dt / r * (p[c] - p[m]) * P.dyi;
                    }
                    if (k >= 2) {
                        const size_t m = id(i, j, k - 1);
                        const T r = T(0.5) * (rho[c] + rho[m]);
                        w[c] = ws[c] - P.dt / r * (p[c] - p[m]) * P.dzi;
                    }
                }
    }

    // set_bc_vel_{j,i,k}_kernel in the order of apply_bc_velocity
    // (voftrial1.cu:959-1051, 1107-1120).
    void bc_velocity() {
        const int jb = 0, jt = P.ny + 1, ib = 0, ir = P.nx + 1, kb = 0, kf = P.nz + 1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 0; k < NZ; ++k)
            for (int i = 0; i < NX; ++i) {
                u[id(i, jb, k)] = u[id(i, 1, k)];
                v[id(i, 1, k)] = T(0);
                w[id(i, jb, k)] = w[id(i, 1, k)];
                u[id(i, jt, k)] = u[id(i, P.ny, k)];
                v[id(i, jt, k)] = T(0);
                w[id(i, jt, k)] = w[id(i, P.ny, k)];
            }
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 0; k < NZ; ++k)
            for (int j = 0; j < NY; ++j) {
                u[id(1, j, k)] = T(0);
                v[id(ib, j, k)] = v[id(1, j, k)];
                w[id(ib, j, k)] = w[id(1, j, k)];
                u[id(ir, j, k)] = T(0);
                v[id(ir, j, k)] = v[id(P.nx, j, k)];
                w[id(ir, j, k)] = w[id(P.nx, j, k)];
            }
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i) {
                u[id(i, j, kb)] = u[id(i, j, 1)];
                v[id(i, j, kb)] = v[id(i, j, 1)];
                w[id(i, j, 1)] = T(0);
                u[id(i, j, kf)] = u[id(i, j, P.nz)];
                v[id(i, j, kf)] = v[id(i, j, P.nz)];
                w[id(i, j, kf)] = T(0);
            }
    }

    // set_bc_F_{j,i,k}_kernel in the order of apply_bc_F (voftrial1.cu:1053-1135).
    void bc_F() {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 0; k < NZ; ++k)
            for (int i = 0; i < NX; ++i) {
                F[id(i, 0, k)] = F[id(i, 1, k)];
                F[id(i, P.ny + 1, k)] = F[id(i, P.ny, k)];
            }
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 0; k < NZ; ++k)
            for (int j = 0; j < NY; ++j) {
                F[id(0, j, k)] = F[id(1, j, k)];
                F[id(P.nx + 1, j, k)] = F[id(P.nx, j, k)];
            }
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i) {
                F[id(i, j, 0)] = F[id(i, j, 1)];
                F[id(i, j, P.nz + 1)] = F[id(i, j, P.nz)];
            }
    }

    // set_bc_{j,i,k}_kernel (voftrial1.cu:105-228) in the order of apply_bc
    // (voftrial1.cu:943-956): the ghost cells of u, v, w, F, p and rho, and
    // the wall-normal velocity on the first and last faces.  The reference's
    // time loop never calls it.
    void bc_all() {
        const int jb = 0, jt = P.ny + 1, ib = 0, ir = P.nx + 1, kb = 0, kf = P.nz + 1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 0; k < NZ; ++k)
            for (int i = 0; i < NX; ++i) {
                const size_t bg = id(i, jb, k), bi = id(i, 1, k), tg = id(i, jt, k), ti = id(i, P.ny, k);
                u[bg] = u[bi];
                v[bi] = T(0);
                w[bg] = w[bi];
                F[bg] = F[bi];
                p[bg] = p[bi];
                rho[bg] = rho[bi];
                u[tg] = u[ti];
                v[tg] = T(0);
                w[tg] = w[ti];
                F[tg] = F[ti];
                p[tg] = p[ti];
                rho[tg] = rho[ti];
            }
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 0; k < NZ; ++k)
            for (int j = 0; j < NY; ++j) {
                const size_t lg = id(ib, j, k), li = id(1, j, k), rg = id(ir, j, k), ri = id(P.nx, j, k);
                u[li] = T(0);
                v[lg] = v[li];
                w[lg] = w[li];
                F[lg] = F[li];
                p[lg] = p[li];
                rho[lg] = rho[li];
                u[rg] = T(0);
                v[rg] = v[ri];
                w[rg] = w[ri];
                F[rg] = F[ri];
                p[rg] = p[ri];
                rho[rg] = rho[ri];
            }
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i) {
                const size_t bg = id(i, j, kb), bi = id(i, j, 1), fg = id(i, j, kf), fi = id(i, j, P.nz);
                u[bg] = u[bi];
                v[bg] = v[bi];
                w[bi] = T(0);
                F[bg] = F[bi];
                p[bg] = p[bi];
                rho[bg] = rho[bi];
                u[fg] = u[fi];
                v[fg] = v[fi];
                w[fg] = T(0);
                F[fg] = F[fi];
                p[fg] = p[fi];
                rho[fg] = rho[fi];
            }
    }

    // post_process_f_kernel, voftrial1.cu:502-507
    void post_process() {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long long t = 0; t < (long long)N; ++t) F[t] = clamp01s(F[t]);
    }

    // ---- FCT sweeps --------------------------------------------------------
    // One generic sweep over the reference's four stages.  `DIR` is the sweep
    // axis; the unit offsets of the sweep axis (s) and of the paired axis used
    // by the x/y stages follow the reference's kernels:
    //   x: fct_x_sweep_stage1..4, voftrial1.cu:509-646  (a = ax, b = ay)
    //   y: fct_y_sweep_stage1..4, voftrial1.cu:648-785  (a = ay, b = ax)
    //   z: fct_z_sweep_stage1..4, voftrial1.cu:787-905  (a = az only)
    template <int DIR>
    size_t fct_stride() const {
        return DIR == 0 ? (size_t)1 : (DIR == 1 ? (size_t)NX : (size_t)NX * NY);
    }
    template <int DIR>
    T fct_dvfac() const {
        return DIR == 0 ? P.dt * P.dy * P.dz : (DIR == 1 ? P.dt * P.dx * P.dz : P.dt * P.dx * P.dy);
    }
    inline T lowflux(const std::vector<T>& vel, size_t face, size_t cm, size_t cp) {
        const T uf = vel[face];
        return sw.br(uf >= T(0)) ? uf * P.dt * F[cm] : uf * P.dt * F[cp];
    }
    inline T highflux(const std::vector<T>& vel, size_t face, size_t cm, size_t cp) {
        const T uf = vel[face];
        return sw.br(uf <= T(0)) ? uf * P.dt * F[cm] : uf * P.dt * F[cp];
    }
    std::vector<T>& fct_A(int dir) { return dir == 0 ? ax : (dir == 1 ? ay : az); }

    // stage 1 (voftrial1.cu:509-536 / 648-675 / 787-812)
    template <int DIR>
    void fct_stage1(const std::vector<T>& vel) {
        const T vol = P.dx * P.dy * P.dz;
        const size_t s = fct_stride<DIR>();
        const T dvfac = fct_dvfac<DIR>();
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    const T dv = vol - dvfac * (vel[c + s] - vel[c]);
                    const T f_in = lowflux(vel, c, c - s, c);       // flux through the lower face
                    const T f_out = lowflux(vel, c + s, c, c + s);  // flux through the upper face
                    T term;
                    if (DIR == 0) term = (f_in - f_out) * P.dy * P.dz / vol;
                    else if (DIR == 1) term = (f_in - f_out) * P.dy / (P.dx * P.dy);
                    else term = (f_in - f_out) * P.dy * P.dx / vol;
                    T out = (F[c] + term) * vol / dv;
                    if (sw.br(out > T(1) || out < T(0))) out = clamp01s(out);
                    Ftd[c] = out;
                }
    }

    // stage 2 (voftrial1.cu:538-586 / 677-725 / 814-860)
    template <int DIR>
    void fct_stage2(const std::vector<T>& vel) {
        const size_t sx = 1, sy = (size_t)NX, sz = (size_t)NX * NY;
        const size_t s = fct_stride<DIR>();
        const T hq = DIR == 2 ? P.dz : P.dx;
        std::vector<T>& A = fct_A(DIR);
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    const T fmx = sw.mx(Ftd[c], sw.mx(Ftd[c - s], Ftd[c + s]));
                    const T fmn = sw.mn(Ftd[c], sw.mn(Ftd[c - s], Ftd[c + s]));
                    A[c + s] = highflux(vel, c + s, c, c + s) - lowflux(vel, c + s, c, c + s);
                    A[c] = highflux(vel, c, c - s, c) - lowflux(vel, c, c - s, c);
                    T pp, pm;
                    if (DIR == 0) {
                        ay[c + sy] = T(0);
                        ay[c] = T(0);
                        pp = sw.mx(T(0), ax[c]) - sw.mn(T(0), ax[c + sx]) + sw.mx(T(0), ay[c]) -
                             sw.mn(T(0), ay[c + sy]);
                        pm = sw.mx(T(0), ax[c + sx]) - sw.mn(T(0), ax[c]) + sw.mx(T(0), ay[c + sy]) -
                             sw.mn(T(0), ay[c]);
                    } else if (DIR == 1) {
                        ax[c + sx] = T(0);
                        ax[c] = T(0);
                        pp = sw.mx(T(0), ax[c]) - sw.mn(T(0), ax[c + sx]) + sw.mx(T(0), ay[c]) -
                             sw.mn(T(0), ay[c + sy]);
                        pm = sw.mx(T(0), ax[c + sx]) - sw.mn(T(0), ax[c]) + sw.mx(T(0), ay[c + sy]) -
                             sw.mn(T(0), ay[c]);
                    } else {
                        pp = sw.mx(T(0), az[c]) - sw.mn(T(0), az[c + sz]);
                        pm = sw.mx(T(0), az[c + sz]) - sw.mn(T(0), az[c]);
                    }
                    const T qp = (fmx - Ftd[c]) * hq;
                    rp[c] = sw.br(pp > T(0)) ? sw.mn(T(1), qp / pp) : T(0);
                    const T qm = (Ftd[c] - fmn) * hq;
                    rm[c] = sw.br(pm > T(0)) ? sw.mn(T(1), qm / pm) : T(0);
                }
    }

    // stage 3 (voftrial1.cu:588-617 / 727-756 / 862-879)
    template <int DIR>
    void fct_stage3() {
        const size_t sx = 1, sy = (size_t)NX, sz = (size_t)NX * NY;
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    if (DIR == 2) {
                        cz[c + sz] = sw.br(az[c + sz] >= T(0)) ? sw.mn(rp[c + sz], rm[c]) : sw.mn(rp[c], rm[c + sz]);
                    } else {
                        cx[c + sx] = sw.br(ax[c + sx] >= T(0)) ? sw.mn(rp[c + sx], rm[c]) : sw.mn(rp[c], rm[c + sx]);
                        cy[c + sy] = sw.br(ay[c + sy] >= T(0)) ? sw.mn(rp[c + sy], rm[c]) : sw.mn(rp[c], rm[c + sy]);
                    }
                }
    }

    // The stage-4 value before its clamp at interior cell c.
    template <int DIR>
    inline T fct_stage4_out(const std::vector<T>& vel, size_t c) const {
        const size_t sx = 1, sy = (size_t)NX, sz = (size_t)NX * NY;
        const T vol = P.dx * P.dy * P.dz;
        const size_t s = fct_stride<DIR>();
        const T dv = vol - fct_dvfac<DIR>() * (vel[c + s] - vel[c]);
        if (DIR == 2) return Ftd[c] - ((az[c + sz] * cz[c + sz] - az[c] * cz[c]) / P.dz) * vol / dv;
        return Ftd[c] -
               ((ax[c + sx] * cx[c + sx] - ax[c] * cx[c] + ay[c + sy] * cy[c + sy] - ay[c] * cy[c]) / P.dy) * vol /
                   dv;
    }

    // stage 4 (voftrial1.cu:619-646 / 758-785 / 881-905)
    template <int DIR>
    void fct_stage4(const std::vector<T>& vel) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    F[c] = clamp01s(fct_stage4_out<DIR>(vel, c));
                }
    }

    template <int DIR>
    void fct_sweep(const std::vector<T>& vel) {
        fct_stage1<DIR>(vel);
        fct_stage2<DIR>(vel);
        fct_stage3<DIR>();
        fct_stage4<DIR>(vel);
    }

    // Convergent pressure solve (extension; no reference counterpart):
    // A p = rhs - mean(rhs) with the Jacobi sweep's Neumann operator, by
    // conjugate gradients on -A from the current p, to ||r|| <= tol ||b||,
    // then the gauge mean(p) = 0.  Returns the final relative residual.
    double conv_tol = 0.0;  // > 0 selects the convergent solve
    int conv_iters = 0;
    void apply_negA(const std::vector<double>& x, std::vector<double>& y) {
        const double cx = (double)P.dxi * P.dxi, cyy = (double)P.dyi * P.dyi, cz = (double)P.dzi * P.dzi;
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    const double xc = x[c];
                    double s = 0;
                    if (i != P.nx) s += cx * (x[id(i + 1, j, k)] - xc);
                    if (i != 1) s += cx * (x[id(i - 1, j, k)] - xc);
                    if (j != P.ny) s += cyy * (x[id(i, j + 1, k)] - xc);
                    if (j != 1) s += cyy * (x[id(i, j - 1, k)] - xc);
                    if (k != P.nz) s += cz * (x[id(i, j, k + 1)] - xc);
                    if (k != 1) s += cz * (x[id(i, j, k - 1)] - xc);
                    y[c] = -s;
                }
    }
    double dot_in(const std::vector<double>& a, const std::vector<double>& b) {
        double s = 0;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(+ : s)
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) s += a[id(i, j, k)] * b[id(i, j, k)];
        return s;
    }
    double solve_conv() {
        const size_t n = N;
        std::vector<double> x(n, 0.0), b(n, 0.0), r(n, 0.0), d(n, 0.0), q(n, 0.0);
        double mean = 0;
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) {
                    x[id(i, j, k)] = (double)p[id(i, j, k)];
                    b[id(i, j, k)] = (double)rhs_at(i, j, k);
                    mean += b[id(i, j, k)];
                }
        const double ncell = (double)P.nx * P.ny * P.nz;
        mean /= ncell;
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) b[id(i, j, k)] = -(b[id(i, j, k)] - mean);  // system -A x = -b
        apply_negA(x, q);
        for (size_t t = 0; t < n; ++t) r[t] = b[t] - q[t];
        const double bn = std::sqrt(dot_in(b, b));
        double rr = dot_in(r, r);
        d = r;
        int it = 0;
        while (bn > 0 && std::sqrt(rr) > conv_tol * bn && it < 20000) {
            apply_negA(d, q);
            const double al = rr / dot_in(d, q);
            for (size_t t = 0; t < n; ++t) {
                x[t] += al * d[t];
                r[t] -= al * q[t];
            }
            const double rr2 = dot_in(r, r);
            for (size_t t = 0; t < n; ++t) d[t] = r[t] + (rr2 / rr) * d[t];
            rr = rr2;
            ++it;
        }
        conv_iters = it;
        double pm = 0;
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) pm += x[id(i, j, k)];
        pm /= ncell;
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) p[id(i, j, k)] = (T)(x[id(i, j, k)] - pm);
        return bn > 0 ? std::sqrt(rr) / bn : 0.0;
    }

    // One time step, voftrial1.cu:1364-1401.
    void step(int istep) {
        cal_nu_rho();
        advect_u();
        advect_v();
        advect_w();
        if (conv_tol > 0) {
            if constexpr (std::is_floating_point<T>::value) solve_conv();
        } else {
            for (int it = 0; it < P.jacobi_iters; ++it) {
                jacobi_sweep(p, pt);
                std::swap(p, pt);
            }
        }
        update_uvw();
        bc_velocity();
        const int r = ((istep % 3) + 3) % 3;
        if (r == 0) { fct_sweep<0>(u); fct_sweep<1>(v); fct_sweep<2>(w); }
        else if (r == 1) { fct_sweep<1>(v); fct_sweep<2>(w); fct_sweep<0>(u); }
        else { fct_sweep<2>(w); fct_sweep<0>(u); fct_sweep<1>(v); }
        post_process();
        bc_F();
    }

    void rhs_field(std::vector<T>& out) {
        out.assign(N, T(0));
        for (int k = 1; k <= P.nz; ++k)
            for (int j = 1; j <= P.ny; ++j)
                for (int i = 1; i <= P.nx; ++i) out[id(i, j, k)] = rhs_at(i, j, k);
    }
};


}  // namespace vofo
