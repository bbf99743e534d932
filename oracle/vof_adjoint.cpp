// vof_adjoint.cpp -- FP64 host adjoint of the voftrial1.cu time step, the
// dual-number tangent it is the transpose of, and the switch tape.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/ (and bench.py's CPU leg) as the
// oracle of the CUDA adjoint (vof_forward_record / vof_backward); the
// product never links or calls it.  The reference has no adjoint: this is the
// reverse mode of the step in oracle_core.h, kernel by kernel
// (voftrial1.cu:1364-1401 backwards), with every non-smooth choice frozen at
// the base point as the forward took it:
//   upwinding (voftrial1.cu:267-275 and the v/w twins): the branch taken;
//   fmax / fmin (FCT stage 2/3, voftrial1.cu:554-557, 580, 585, 606-616): the
//     argument returned, the first one on a tie;
//   clamps (median3, voftrial1.cu:52-60; the stage-1 range test): derivative 1
//     for a value in [0, 1], 0 outside.
// The tangent-linear forward (Dual below) takes the same choices, so
// <adjoint, d> equals its directional derivative to rounding (the transpose
// test); the tangent itself is checked against central differences of the
// unfrozen FP64 forward.  Taped (oracle_core.h) records the choices of a run
// and can replay them (a frozen-switch forward).
//
// Loss: L = sum of F dV over the interior cells whose centre
// ((i - 1/2) dx, (j - 1/2) dy, (k - 1/2) dz) lies strictly inside a box.
// Outputs: dL/d(F, u, v, w, p) of the initial state (reference layout, every
// entry) and dL/d(gx, gy, gz).  The forward runs in T (float: the FP32 path,
// bit for bit; double: the FP64 oracle); every adjoint quantity is double.
#include "oracle_core.h"

namespace {
using namespace vofo;

struct Box {
    double x0, x1, y0, y1, z0, z1;
};

template <typename T, typename SW>
bool in_box(const Oracle<T, SW>& o, const Box& b, int i, int j, int k) {
    const double xc = (i - 0.5) * (double)o.P.dx, yc = (j - 0.5) * (double)o.P.dy, zc = (k - 0.5) * (double)o.P.dz;
    return xc > b.x0 && xc < b.x1 && yc > b.y0 && yc < b.y1 && zc > b.z0 && zc < b.z1;
}

template <typename T, typename SW>
double box_loss(const Oracle<T, SW>& o, const Box& b) {
    const double dV = (double)o.P.dx * (double)o.P.dy * (double)o.P.dz;
    double L = 0;
    for (int k = 1; k <= o.P.nz; ++k)
        for (int j = 1; j <= o.P.ny; ++j)
            for (int i = 1; i <= o.P.nx; ++i)
                if (in_box(o, b, i, j, k)) L += (double)o.F[o.id(i, j, k)] * dV;
    return L;
}

// The sweep axes of step istep (voftrial1.cu:1389-1397).
inline void sweep_order(int istep, int dirs[3]) {
    const int r = ((istep % 3) + 3) % 3;
    const int o[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
    for (int q = 0; q < 3; ++q) dirs[q] = o[r][q];
}

template <typename T>
struct State {
    std::vector<T> F, u, v, w, p;
};

inline double dclamp(double v) { return (v >= 0.0 && v <= 1.0) ? 1.0 : 0.0; }

template <typename T>
struct Adjoint {
    Oracle<T> o;
    std::vector<double> lF, lu, lv, lw, lp;        // adjoint of the state
    std::vector<double> lus, lvs, lws, lrho, lnu, lrhs, lq, lFn;
    std::vector<double> lFtd, lA, lC, lrp, lrm, ldv;  // of one sweep
    double lg[3] = {0, 0, 0};
    double conv_tol = 0.0;  // > 0: the pressure is the convergent solve (oracle_core.h solve_conv)
    // forward values of the step being reversed
    std::vector<T> rho, nu, us, vs, ws, pafter, u1, v1, w1, Fin[3], Fstart, ustart, vstart, wstart;

    Adjoint(const Prm<T>& P, int nth) : o(P, nth) {
        for (auto* f : {&lF, &lu, &lv, &lw, &lp, &lus, &lvs, &lws, &lrho, &lnu, &lrhs, &lq, &lFn, &lFtd, &lA, &lC,
                        &lrp, &lrm, &ldv})
            f->assign(o.N, 0.0);
    }
    size_t id(int i, int j, int k) const { return o.id(i, j, k); }

    // ---- forward values of step `istep` from its start state --------------
    void recompute(const State<T>& S, int istep) {
        o.F = S.F;
        o.u = S.u;
        o.v = S.v;
        o.w = S.w;
        o.p = S.p;
        Fstart = S.F;
        ustart = S.u;
        vstart = S.v;
        wstart = S.w;
        o.cal_nu_rho();
        rho = o.rho;
        nu = o.nu;
        o.advect_u();
        o.advect_v();
        o.advect_w();
        us = o.us;
        vs = o.vs;
        ws = o.ws;
        if (conv_tol > 0) {
            o.conv_tol = conv_tol;
            o.solve_conv();
        } else {
            for (int it = 0; it < o.P.jacobi_iters; ++it) {
                o.jacobi_sweep(o.p, o.pt);
                std::swap(o.p, o.pt);
            }
        }
        pafter = o.p;
        o.update_uvw();
        o.bc_velocity();
        u1 = o.u;
        v1 = o.v;
        w1 = o.w;
        int dirs[3];
        sweep_order(istep, dirs);
        for (int q = 0; q < 3; ++q) {
            Fin[q] = o.F;
            if (dirs[q] == 0) o.template fct_sweep<0>(u1);
            else if (dirs[q] == 1) o.template fct_sweep<1>(v1);
            else o.template fct_sweep<2>(w1);
        }
    }

    // ---- F boundary copies (set_bc_F_*, voftrial1.cu:1053-1135), reversed --
    void adj_bc_F() {
        const int NX = o.NX, NY = o.NY, NZ = o.NZ, nx = o.P.nx, ny = o.P.ny, nz = o.P.nz;
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i) {
                lF[id(i, j, 1)] += lF[id(i, j, 0)];
                lF[id(i, j, 0)] = 0;
                lF[id(i, j, nz)] += lF[id(i, j, nz + 1)];
                lF[id(i, j, nz + 1)] = 0;
            }
        for (int k = 0; k < NZ; ++k)
            for (int j = 0; j < NY; ++j) {
                lF[id(1, j, k)] += lF[id(0, j, k)];
                lF[id(0, j, k)] = 0;
                lF[id(nx, j, k)] += lF[id(nx + 1, j, k)];
                lF[id(nx + 1, j, k)] = 0;
            }
        for (int k = 0; k < NZ; ++k)
            for (int i = 0; i < NX; ++i) {
                lF[id(i, 1, k)] += lF[id(i, 0, k)];
                lF[id(i, 0, k)] = 0;
                lF[id(i, ny, k)] += lF[id(i, ny + 1, k)];
                lF[id(i, ny + 1, k)] = 0;
            }
    }

    // ---- one FCT sweep (voftrial1.cu:509-905), reversed ---------------------
    // In: lF = adjoint of F after the sweep.  Out: lF = adjoint of F before it;
    // lvel += adjoint of the face velocities.
    template <int DIR>
    void adj_sweep(const std::vector<T>& Fsweep, const std::vector<T>& vel, std::vector<double>& lvel) {
        const size_t s = o.template fct_stride<DIR>();
        o.F = Fsweep;
        o.template fct_stage1<DIR>(vel);
        o.template fct_stage2<DIR>(vel);
        o.template fct_stage3<DIR>();
        const std::vector<T>& F = Fsweep;
        const std::vector<T>& A = o.fct_A(DIR);
        const std::vector<T>& Cc = DIR == 0 ? o.cx : (DIR == 1 ? o.cy : o.cz);
        const std::vector<T>& Ftd = o.Ftd;
        const double dt = o.P.dt, vol = (double)(o.P.dx * o.P.dy * o.P.dz);
        const double dvfac = (double)o.template fct_dvfac<DIR>();
        const double hq = DIR == 2 ? (double)o.P.dz : (double)o.P.dx;
        const double K4 = DIR == 2 ? (double)o.P.dz : (double)o.P.dy;
        const double K1 = DIR == 0 ? (double)o.P.dy * o.P.dz / vol
                                   : (DIR == 1 ? (double)o.P.dy / ((double)o.P.dx * o.P.dy)
                                               : (double)o.P.dy * o.P.dx / vol);
        const T volT = o.P.dx * o.P.dy * o.P.dz;
        const T dvfacT = o.template fct_dvfac<DIR>();
        for (auto* f : {&lFtd, &lA, &lC, &lrp, &lrm, &ldv}) std::fill(f->begin(), f->end(), 0.0);
        // the new lF: ghosts pass through (the sweep leaves them), interior rebuilt
        lFn = lF;
        const int nx = o.P.nx, ny = o.P.ny, nz = o.P.nz;
        const int nlast = DIR == 0 ? nx : (DIR == 1 ? ny : nz);
        auto axis_pos = [&](int i, int j, int k) { return DIR == 0 ? i : (DIR == 1 ? j : k); };
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) lFn[id(i, j, k)] = 0.0;
        // stage 4
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    const size_t c = id(i, j, k);
                    const double out = (double)o.template fct_stage4_out<DIR>(vel, c);
                    const double g = lF[c] * dclamp(out);
                    if (g == 0.0) continue;
                    lFtd[c] += g;
                    const double dv = (double)(volT - dvfacT * (vel[c + s] - vel[c]));
                    const double X = ((double)A[c + s] * Cc[c + s] - (double)A[c] * Cc[c]) / K4;
                    const double lX = -g * vol / dv;
                    ldv[c] += g * X * vol / (dv * dv);
                    lA[c + s] += lX * Cc[c + s] / K4;
                    lC[c + s] += lX * A[c + s] / K4;
                    lA[c] -= lX * Cc[c] / K4;
                    lC[c] -= lX * A[c] / K4;
                }
        // stage 3: face c+s of every interior cell c
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    const size_t c = id(i, j, k);
                    const double g = lC[c + s];
                    if (g == 0.0) continue;
                    if (A[c + s] >= T(0)) {
                        if (o.rp[c + s] <= o.rm[c]) lrp[c + s] += g;
                        else lrm[c] += g;
                    } else {
                        if (o.rp[c] <= o.rm[c + s]) lrp[c] += g;
                        else lrm[c + s] += g;
                    }
                }
        // stage 2: limiter ratios and the local extrema
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    const size_t c = id(i, j, k);
                    const T a0 = A[c], a1 = A[c + s];
                    T pp, pm;
                    {   // the same float expressions as stage 2 (the cross-axis terms are zero)
                        pp = std::fmax(T(0), a0) - std::fmin(T(0), a1);
                        pm = std::fmax(T(0), a1) - std::fmin(T(0), a0);
                        if (DIR != 2) {
                            pp = pp + std::fmax(T(0), T(0)) - std::fmin(T(0), T(0));
                            pm = pm + std::fmax(T(0), T(0)) - std::fmin(T(0), T(0));
                        }
                    }
                    const T fmx = std::fmax(Ftd[c], std::fmax(Ftd[c - s], Ftd[c + s]));
                    const T fmn = std::fmin(Ftd[c], std::fmin(Ftd[c - s], Ftd[c + s]));
                    const T qp = (fmx - Ftd[c]) * (DIR == 2 ? o.P.dz : o.P.dx);
                    const T qm = (Ftd[c] - fmn) * (DIR == 2 ? o.P.dz : o.P.dx);
                    double lqp = 0, lqm = 0, lpp = 0, lpm = 0;
                    if (lrp[c] != 0.0 && pp > T(0) && qp / pp < T(1)) {
                        lqp = lrp[c] / (double)pp;
                        lpp = -lrp[c] * (double)qp / ((double)pp * pp);
                    }
                    if (lrm[c] != 0.0 && pm > T(0) && qm / pm < T(1)) {
                        lqm = lrm[c] / (double)pm;
                        lpm = -lrm[c] * (double)qm / ((double)pm * pm);
                    }
                    if (lqp != 0.0) {
                        const double lfmx = lqp * hq;
                        lFtd[c] -= lqp * hq;
                        const size_t in = (Ftd[c - s] >= Ftd[c + s]) ? c - s : c + s;
                        const size_t sel = (Ftd[c] >= Ftd[in]) ? c : in;
                        lFtd[sel] += lfmx;
                    }
                    if (lqm != 0.0) {
                        const double lfmn = -lqm * hq;
                        lFtd[c] += lqm * hq;
                        const size_t in = (Ftd[c - s] <= Ftd[c + s]) ? c - s : c + s;
                        const size_t sel = (Ftd[c] <= Ftd[in]) ? c : in;
                        lFtd[sel] += lfmn;
                    }
                    if (a0 > T(0)) lA[c] += lpp;
                    if (a1 < T(0)) lA[c + s] -= lpp;
                    if (a1 > T(0)) lA[c + s] += lpm;
                    if (a0 < T(0)) lA[c] -= lpm;
                }
        // antidiffusive fluxes A = highflux - lowflux at every face of the line
        auto adj_face = [&](size_t f) {
            const double g = lA[f];
            if (g == 0.0) return;
            const T uf = vel[f];
            const size_t hs = (uf <= T(0)) ? f - s : f;
            const size_t ls = (uf >= T(0)) ? f - s : f;
            lvel[f] += g * dt * ((double)F[hs] - (double)F[ls]);
            lFn[hs] += g * (double)uf * dt;
            lFn[ls] -= g * (double)uf * dt;
        };
        // stage 1
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    const size_t c = id(i, j, k);
                    adj_face(c);
                    if (axis_pos(i, j, k) == nlast) adj_face(c + s);
                    const T dvT = volT - dvfacT * (vel[c + s] - vel[c]);
                    const size_t lin = (vel[c] >= T(0)) ? c - s : c;
                    const size_t lout = (vel[c + s] >= T(0)) ? c : c + s;
                    const T f_in = vel[c] * o.P.dt * F[lin];
                    const T f_out = vel[c + s] * o.P.dt * F[lout];
                    T term;
                    if (DIR == 0) term = (f_in - f_out) * o.P.dy * o.P.dz / volT;
                    else if (DIR == 1) term = (f_in - f_out) * o.P.dy / (o.P.dx * o.P.dy);
                    else term = (f_in - f_out) * o.P.dy * o.P.dx / volT;
                    const T out = (F[c] + term) * volT / dvT;
                    const double h = (out > T(1) || out < T(0)) ? 0.0 : lFtd[c];
                    const double dv = (double)dvT;
                    if (h != 0.0) {
                        lFn[c] += h * vol / dv;
                        const double lterm = h * vol / dv;
                        ldv[c] -= h * ((double)F[c] + (double)term) * vol / (dv * dv);
                        const double lfin = lterm * K1, lfout = -lterm * K1;
                        lvel[c] += lfin * dt * (double)F[lin];
                        lFn[lin] += lfin * (double)vel[c] * dt;
                        lvel[c + s] += lfout * dt * (double)F[lout];
                        lFn[lout] += lfout * (double)vel[c + s] * dt;
                    }
                    // dv = vol - dvfac (vel[c+s] - vel[c]) (stages 1 and 4)
                    lvel[c + s] -= ldv[c] * dvfac;
                    lvel[c] += ldv[c] * dvfac;
                }
        lF.swap(lFn);
    }

    // ---- set_bc_vel_* (voftrial1.cu:959-1051), reversed ------------------------
    void adj_bc_velocity() {
        const int NX = o.NX, NY = o.NY, NZ = o.NZ, nx = o.P.nx, ny = o.P.ny, nz = o.P.nz;
        auto mv = [](std::vector<double>& l, size_t dst, size_t src) {
            l[src] += l[dst];
            l[dst] = 0;
        };
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i) {
                mv(lu, id(i, j, 0), id(i, j, 1));
                mv(lv, id(i, j, 0), id(i, j, 1));
                lw[id(i, j, 1)] = 0;
                mv(lu, id(i, j, nz + 1), id(i, j, nz));
                mv(lv, id(i, j, nz + 1), id(i, j, nz));
                lw[id(i, j, nz + 1)] = 0;
            }
        for (int k = 0; k < NZ; ++k)
            for (int j = 0; j < NY; ++j) {
                lu[id(1, j, k)] = 0;
                mv(lv, id(0, j, k), id(1, j, k));
                mv(lw, id(0, j, k), id(1, j, k));
                lu[id(nx + 1, j, k)] = 0;
                mv(lv, id(nx + 1, j, k), id(nx, j, k));
                mv(lw, id(nx + 1, j, k), id(nx, j, k));
            }
        for (int k = 0; k < NZ; ++k)
            for (int i = 0; i < NX; ++i) {
                mv(lu, id(i, 0, k), id(i, 1, k));
                lv[id(i, 1, k)] = 0;
                mv(lw, id(i, 0, k), id(i, 1, k));
                mv(lu, id(i, ny + 1, k), id(i, ny, k));
                lv[id(i, ny + 1, k)] = 0;
                mv(lw, id(i, ny + 1, k), id(i, ny, k));
            }
    }

    // ---- update_{u,v,w}_kernel (voftrial1.cu:441-493), reversed -------------
    void adj_update() {
        const double dt = o.P.dt;
        const double hinv[3] = {(double)o.P.dxi, (double)o.P.dyi, (double)o.P.dzi};
        const size_t st[3] = {1, (size_t)o.NX, (size_t)o.NX * o.NY};
        std::vector<double>* lvel[3] = {&lu, &lv, &lw};
        std::vector<double>* lvs_[3] = {&lus, &lvs, &lws};
        for (int k = 1; k <= o.P.nz; ++k)
            for (int j = 1; j <= o.P.ny; ++j)
                for (int i = 1; i <= o.P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    const int pos[3] = {i, j, k};
                    for (int a = 0; a < 3; ++a) {
                        if (pos[a] < 2) continue;
                        const size_t m = c - st[a];
                        const double g = (*lvel[a])[c];
                        (*lvel[a])[c] = 0;
                        if (g == 0.0) continue;
                        const T rT = T(0.5) * (rho[c] + rho[m]);
                        const double r = (double)rT;
                        (*lvs_[a])[c] += g;
                        const double coef = dt / r * hinv[a];
                        lp[c] -= g * coef;
                        lp[m] += g * coef;
                        const double lr = g * dt * ((double)pafter[c] - (double)pafter[m]) * hinv[a] / (r * r);
                        lrho[c] += 0.5 * lr;
                        lrho[m] += 0.5 * lr;
                    }
                }
    }

    // ---- the Jacobi sweeps (voftrial1.cu:401-439), transposed ------------------
    // p' = (rhs - N p) / ap: lambda -> mu = lambda / ap, lrhs += mu, lambda' = -N mu.
    void adj_jacobi() {
        const double cxx = (double)(o.P.dxi * o.P.dxi), cyy = (double)(o.P.dyi * o.P.dyi),
                     czz = (double)(o.P.dzi * o.P.dzi);
        const int nx = o.P.nx, ny = o.P.ny, nz = o.P.nz;
        std::vector<double>& mu = lq;
        for (int it = 0; it < o.P.jacobi_iters; ++it) {
            std::fill(mu.begin(), mu.end(), 0.0);
            for (int k = 1; k <= nz; ++k)
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i) {
                        const T ae = (i != nx) ? o.P.dxi * o.P.dxi : T(0), aw = (i != 1) ? o.P.dxi * o.P.dxi : T(0);
                        const T an = (j != ny) ? o.P.dyi * o.P.dyi : T(0), as = (j != 1) ? o.P.dyi * o.P.dyi : T(0);
                        const T af = (k != nz) ? o.P.dzi * o.P.dzi : T(0), ab = (k != 1) ? o.P.dzi * o.P.dzi : T(0);
                        const T ap = -(ae + aw + an + as + af + ab);
                        const size_t c = id(i, j, k);
                        mu[c] = lp[c] / (double)ap;
                        lrhs[c] += mu[c];
                    }
            for (int k = 1; k <= nz; ++k)
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i) {
                        const size_t c = id(i, j, k);
                        double s = 0;
                        if (i != nx) s += cxx * mu[id(i + 1, j, k)];
                        if (i != 1) s += cxx * mu[id(i - 1, j, k)];
                        if (j != ny) s += cyy * mu[id(i, j + 1, k)];
                        if (j != 1) s += cyy * mu[id(i, j - 1, k)];
                        if (k != nz) s += czz * mu[id(i, j, k + 1)];
                        if (k != 1) s += czz * mu[id(i, j, k - 1)];
                        lp[c] = -s;
                    }
        }
    }

    // ---- the convergent pressure solve, reversed ----------------------------------
    // p = P A+ Q rhs (Q: remove the mean of rhs, P: gauge mean(p) = 0, A the
    // symmetric Neumann operator): lrhs = Q A+ P lp, i.e. the mean-free mu
    // with A mu = lp - mean(lp); the state pressure (a warm start) gets none.
    void adj_solve() {
        const int nx = o.P.nx, ny = o.P.ny, nz = o.P.nz;
        const double ncell = (double)nx * ny * nz;
        std::vector<double> b(o.N, 0.0), x(o.N, 0.0), r(o.N, 0.0), d(o.N, 0.0), q(o.N, 0.0);
        double mean = 0;
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) mean += lp[id(i, j, k)];
        mean /= ncell;
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) b[id(i, j, k)] = -(lp[id(i, j, k)] - mean);  // -A x = -b
        r = b;
        d = r;
        const double bn = std::sqrt(o.dot_in(b, b));
        double rr = o.dot_in(r, r);
        for (int it = 0; bn > 0 && std::sqrt(rr) > 1e-14 * bn && it < 20000; ++it) {
            o.apply_negA(d, q);
            const double al = rr / o.dot_in(d, q);
            for (size_t t = 0; t < o.N; ++t) {
                x[t] += al * d[t];
                r[t] -= al * q[t];
            }
            const double rr2 = o.dot_in(r, r);
            for (size_t t = 0; t < o.N; ++t) d[t] = r[t] + (rr2 / rr) * d[t];
            rr = rr2;
        }
        double xm = 0;
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) xm += x[id(i, j, k)];
        xm /= ncell;
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) lrhs[id(i, j, k)] = x[id(i, j, k)] - xm;
        std::fill(lp.begin(), lp.end(), 0.0);
    }

    // ---- rhs = rho/dt div(u*) (voftrial1.cu:418-422), reversed ----------------
    void adj_rhs() {
        const double dt = o.P.dt, dxi = o.P.dxi, dyi = o.P.dyi, dzi = o.P.dzi;
        const size_t sy = o.NX, sz = (size_t)o.NX * o.NY;
        for (int k = 1; k <= o.P.nz; ++k)
            for (int j = 1; j <= o.P.ny; ++j)
                for (int i = 1; i <= o.P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    const double g = lrhs[c];
                    lrhs[c] = 0;
                    if (g == 0.0) continue;
                    const double div = ((double)us[c + 1] - us[c]) * dxi + ((double)vs[c + sy] - vs[c]) * dyi +
                                       ((double)ws[c + sz] - ws[c]) * dzi;
                    lrho[c] += g * div / dt;
                    const double kk = g * (double)rho[c] / dt;
                    lus[c + 1] += kk * dxi;
                    lus[c] -= kk * dxi;
                    lvs[c + sy] += kk * dyi;
                    lvs[c] -= kk * dyi;
                    lws[c + sz] += kk * dzi;
                    lws[c] -= kk * dzi;
                }
    }

    // ---- advect_{u,v,w}_kernel (voftrial1.cu:230-399), reversed --------------
    // One component: q* = q + dt (visc + adv + g), adv = -a dqdx - b dqdy - c dqdz
    // with the upwind choices by the sign of (a, b, c).
    void adj_advect_comp(int comp) {
        const double dt = o.P.dt;
        const double hx = o.P.dxi, hy = o.P.dyi, hz = o.P.dzi;
        const double hx2 = (double)o.P.dxi * o.P.dxi, hy2 = (double)o.P.dyi * o.P.dyi,
                     hz2 = (double)o.P.dzi * o.P.dzi;
        const size_t sx = 1, sy = o.NX, sz = (size_t)o.NX * o.NY;
        const std::vector<T>& q = comp == 0 ? ustart : (comp == 1 ? vstart : wstart);
        std::vector<double>& lq_ = comp == 0 ? lu : (comp == 1 ? lv : lw);
        std::vector<double>& lqs = comp == 0 ? lus : (comp == 1 ? lvs : lws);
        const int i0 = comp == 0 ? 2 : 1, j0 = comp == 1 ? 2 : 1, k0 = comp == 2 ? 2 : 1;
        for (int k = k0; k <= o.P.nz; ++k)
            for (int j = j0; j <= o.P.ny; ++j)
                for (int i = i0; i <= o.P.nx; ++i) {
                    const size_t c = id(i, j, k);
                    const double G = lqs[c];
                    if (G == 0.0) continue;
                    // advecting velocities (the same float expressions as the forward)
                    T a, b, cc;
                    size_t ia[4], ib[4];  // the entries averaged into the two interpolated ones
                    std::vector<double>*la, *lb;
                    if (comp == 0) {
                        ia[0] = id(i - 1, j, k); ia[1] = id(i - 1, j + 1, k); ia[2] = id(i, j, k); ia[3] = id(i, j + 1, k);
                        ib[0] = id(i - 1, j, k); ib[1] = id(i - 1, j, k + 1); ib[2] = id(i, j, k); ib[3] = id(i, j, k + 1);
                        a = q[c];
                        b = T(0.25) * (vstart[ia[0]] + vstart[ia[1]] + vstart[ia[2]] + vstart[ia[3]]);
                        cc = T(0.25) * (wstart[ib[0]] + wstart[ib[1]] + wstart[ib[2]] + wstart[ib[3]]);
                        la = &lv;
                        lb = &lw;
                    } else if (comp == 1) {
                        ia[0] = id(i, j - 1, k); ia[1] = id(i, j, k); ia[2] = id(i + 1, j - 1, k); ia[3] = id(i + 1, j, k);
                        ib[0] = id(i, j - 1, k + 1); ib[1] = id(i, j - 1, k); ib[2] = id(i, j, k); ib[3] = id(i, j, k + 1);
                        a = T(0.25) * (ustart[ia[0]] + ustart[ia[1]] + ustart[ia[2]] + ustart[ia[3]]);
                        b = q[c];
                        cc = T(0.25) * (wstart[ib[0]] + wstart[ib[1]] + wstart[ib[2]] + wstart[ib[3]]);
                        la = &lu;
                        lb = &lw;
                    } else {
                        ia[0] = id(i + 1, j, k - 1); ia[1] = id(i, j, k - 1); ia[2] = id(i + 1, j, k); ia[3] = id(i, j, k);
                        ib[0] = id(i, j + 1, k - 1); ib[1] = id(i, j, k - 1); ib[2] = id(i, j, k); ib[3] = id(i, j + 1, k);
                        a = T(0.25) * (ustart[ia[0]] + ustart[ia[1]] + ustart[ia[2]] + ustart[ia[3]]);
                        b = T(0.25) * (vstart[ib[0]] + vstart[ib[1]] + vstart[ib[2]] + vstart[ib[3]]);
                        cc = q[c];
                        la = &lu;
                        lb = &lv;
                    }
                    const double qc = q[c], qxm = q[c - sx], qxp = q[c + sx], qym = q[c - sy], qyp = q[c + sy],
                                 qzm = q[c - sz], qzp = q[c + sz];
                    const bool ux = a > T(0), uy = b > T(0), uz = cc > T(0);
                    const double dqdx = ux ? (qc - qxm) * hx : (qxp - qc) * hx;
                    const double dqdy = uy ? (qc - qym) * hy : (qyp - qc) * hy;
                    const double dqdz = uz ? (qc - qzm) * hz : (qzp - qc) * hz;
                    const double Gd = G * dt;
                    const double n_ = nu[c];
                    lg[comp] += Gd;
                    lq_[c] += G;  // q* = q + ...
                    lnu[c] += Gd * ((qxm - 2 * qc + qxp) * hx2 + (qym - 2 * qc + qyp) * hy2 + (qzm - 2 * qc + qzp) * hz2);
                    lq_[c - sx] += Gd * n_ * hx2;
                    lq_[c + sx] += Gd * n_ * hx2;
                    lq_[c - sy] += Gd * n_ * hy2;
                    lq_[c + sy] += Gd * n_ * hy2;
                    lq_[c - sz] += Gd * n_ * hz2;
                    lq_[c + sz] += Gd * n_ * hz2;
                    lq_[c] -= Gd * n_ * 2.0 * (hx2 + hy2 + hz2);
                    // -a dqdx
                    const double la_ = -Gd * dqdx, lb_ = -Gd * dqdy, lc_ = -Gd * dqdz;
                    const double ga = -Gd * (double)a, gb = -Gd * (double)b, gc = -Gd * (double)cc;
                    if (ux) { lq_[c] += ga * hx; lq_[c - sx] -= ga * hx; }
                    else { lq_[c + sx] += ga * hx; lq_[c] -= ga * hx; }
                    if (uy) { lq_[c] += gb * hy; lq_[c - sy] -= gb * hy; }
                    else { lq_[c + sy] += gb * hy; lq_[c] -= gb * hy; }
                    if (uz) { lq_[c] += gc * hz; lq_[c - sz] -= gc * hz; }
                    else { lq_[c + sz] += gc * hz; lq_[c] -= gc * hz; }
                    // the advecting velocities: the own component directly, the others averaged
                    if (comp == 0) {
                        lu[c] += la_;
                        for (int t = 0; t < 4; ++t) { (*la)[ia[t]] += 0.25 * lb_; (*lb)[ib[t]] += 0.25 * lc_; }
                    } else if (comp == 1) {
                        lv[c] += lb_;
                        for (int t = 0; t < 4; ++t) { (*la)[ia[t]] += 0.25 * la_; (*lb)[ib[t]] += 0.25 * lc_; }
                    } else {
                        lw[c] += lc_;
                        for (int t = 0; t < 4; ++t) { (*la)[ia[t]] += 0.25 * la_; (*lb)[ib[t]] += 0.25 * lb_; }
                    }
                    lqs[c] = 0;
                }
    }

    // ---- cal_nu_rho_kernel (voftrial1.cu:95-104), reversed --------------------
    void adj_rho_nu() {
        const double drho = (double)o.P.rho_l - (double)o.P.rho_g, dnu = (double)o.P.nu_l - (double)o.P.nu_g;
        for (size_t t = 0; t < o.N; ++t) {
            if (lrho[t] != 0.0 || lnu[t] != 0.0) lF[t] += (lrho[t] * drho + lnu[t] * dnu) * dclamp((double)Fstart[t]);
            lrho[t] = 0;
            lnu[t] = 0;
        }
    }

    // The adjoint of step `istep` from its start state S: (lF, lu, lv, lw, lp)
    // of the state after the step -> of the state before it.
    void step(const State<T>& S, int istep) {
        recompute(S, istep);
        adj_bc_F();
        // post_process leaves the interior unchanged (stage 4 clamped it
        // already) and its ghost values are overwritten by bc_F: nothing to do.
        int dirs[3];
        sweep_order(istep, dirs);
        for (int q = 2; q >= 0; --q) {
            if (dirs[q] == 0) adj_sweep<0>(Fin[q], u1, lu);
            else if (dirs[q] == 1) adj_sweep<1>(Fin[q], v1, lv);
            else adj_sweep<2>(Fin[q], w1, lw);
        }
        adj_bc_velocity();
        adj_update();
        if (conv_tol > 0) adj_solve();
        else adj_jacobi();
        adj_rhs();
        adj_advect_comp(0);
        adj_advect_comp(1);
        adj_advect_comp(2);
        adj_rho_nu();
    }
};

template <typename T>
int adjoint_run(const vof_params* prm, const T* F, const T* u, const T* v, const T* w, const T* p, int istep0,
                int nsteps, const double* box, double* lF, double* lu, double* lv, double* lw, double* lp,
                double* grad_g, double* loss, int nthreads, double conv_tol = 0.0) {
    if (!prm || !F || !u || !v || !w || !p || !box || nsteps < 0) return VOF_E_INVALID;
    if (prm->nx < 1 || prm->ny < 1 || prm->nz < 1) return VOF_E_SIZE;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    const Box b{box[0], box[1], box[2], box[3], box[4], box[5]};
    Adjoint<T> A(make_prm(prm, T(0)), nthreads);
    A.conv_tol = conv_tol;
    Oracle<T>& o = A.o;
    const size_t n = o.N;
    std::vector<State<T>> states((size_t)nsteps);
    State<T> cur{std::vector<T>(F, F + n), std::vector<T>(u, u + n), std::vector<T>(v, v + n),
                 std::vector<T>(w, w + n), std::vector<T>(p, p + n)};
    {
        Oracle<T> fw(make_prm(prm, T(0)), nthreads);
        fw.conv_tol = conv_tol;
        fw.F = cur.F;
        fw.u = cur.u;
        fw.v = cur.v;
        fw.w = cur.w;
        fw.p = cur.p;
        for (int s = 0; s < nsteps; ++s) {
            states[s] = State<T>{fw.F, fw.u, fw.v, fw.w, fw.p};
            fw.step(istep0 + s);
        }
        if (loss) *loss = box_loss(fw, b);
    }
    const double dV = (double)o.P.dx * (double)o.P.dy * (double)o.P.dz;
    for (int k = 1; k <= o.P.nz; ++k)
        for (int j = 1; j <= o.P.ny; ++j)
            for (int i = 1; i <= o.P.nx; ++i)
                if (in_box(o, b, i, j, k)) A.lF[o.id(i, j, k)] = dV;
    for (int s = nsteps - 1; s >= 0; --s) A.step(states[s], istep0 + s);
    std::copy(A.lF.begin(), A.lF.end(), lF);
    std::copy(A.lu.begin(), A.lu.end(), lu);
    std::copy(A.lv.begin(), A.lv.end(), lv);
    std::copy(A.lw.begin(), A.lw.end(), lw);
    std::copy(A.lp.begin(), A.lp.end(), lp);
    if (grad_g)
        for (int q = 0; q < 3; ++q) grad_g[q] = A.lg[q];
    return VOF_OK;
}

// ---- tangent-linear forward (dual numbers) -----------------------------------
// The FP64 step on (value, derivative) pairs: the values are bit for bit the
// FP64 oracle's, the derivatives are J d with the switches decided on the
// values and the first argument winning a tie, i.e. the map the adjoint above
// transposes.  <dL/dx0, d> from the adjoint must equal the loss derivative here.
struct Dual {
    double v = 0, d = 0;
    Dual() = default;
    Dual(double x) : v(x) {}
    Dual(double x, double dx) : v(x), d(dx) {}
    explicit operator double() const { return v; }
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }

struct DualSw {
    static inline bool br(bool c) { return c; }
    static inline Dual mx(Dual a, Dual b) { return a.v >= b.v ? a : b; }
    static inline Dual mn(Dual a, Dual b) { return a.v <= b.v ? a : b; }
};

// Prm<Dual>: the FP64 parameters (make_prm(.., double)), with derivative dg of
// the body force.
inline Prm<Dual> make_prm_dual(const vof_params* p, const double* dg) {
    const Prm<double> q = make_prm(p, 0.0);
    Prm<Dual> r;
    r.nx = q.nx; r.ny = q.ny; r.nz = q.nz;
    r.Lx = q.Lx; r.Ly = q.Ly; r.Lz = q.Lz;
    r.rho_l = q.rho_l; r.rho_g = q.rho_g; r.nu_l = q.nu_l; r.nu_g = q.nu_g;
    r.gx = Dual(q.gx, dg ? dg[0] : 0.0);
    r.gy = Dual(q.gy, dg ? dg[1] : 0.0);
    r.gz = Dual(q.gz, dg ? dg[2] : 0.0);
    r.dt = q.dt;
    r.dx = q.dx; r.dy = q.dy; r.dz = q.dz;
    r.dxi = q.dxi; r.dyi = q.dyi; r.dzi = q.dzi;
    r.jacobi_iters = q.jacobi_iters;
    return r;
}

int tangent_run(const vof_params* prm, const double* x0[5], const double* dx0[5], const double* dg, int istep0,
                int nsteps, const double* box, double* loss, double* dloss, int nthreads) {
    if (!prm || !box || nsteps < 0) return VOF_E_INVALID;
    for (int q = 0; q < 5; ++q)
        if (!x0[q]) return VOF_E_INVALID;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    Oracle<Dual, DualSw> o(make_prm_dual(prm, dg), nthreads);
    std::vector<Dual>* f[5] = {&o.F, &o.u, &o.v, &o.w, &o.p};
    for (int q = 0; q < 5; ++q)
        for (size_t t = 0; t < o.N; ++t) (*f[q])[t] = Dual(x0[q][t], dx0[q] ? dx0[q][t] : 0.0);
    for (int s = 0; s < nsteps; ++s) o.step(istep0 + s);
    const Box b{box[0], box[1], box[2], box[3], box[4], box[5]};
    const double dV = (double)o.P.dx * (double)o.P.dy * (double)o.P.dz;
    double L = 0, dL = 0;
    for (int k = 1; k <= o.P.nz; ++k)
        for (int j = 1; j <= o.P.ny; ++j)
            for (int i = 1; i <= o.P.nx; ++i) {
                const double xc = (i - 0.5) * (double)o.P.dx, yc = (j - 0.5) * (double)o.P.dy,
                             zc = (k - 0.5) * (double)o.P.dz;
                if (xc > b.x0 && xc < b.x1 && yc > b.y0 && yc < b.y1 && zc > b.z0 && zc < b.z1) {
                    L += o.F[o.id(i, j, k)].v * dV;
                    dL += o.F[o.id(i, j, k)].d * dV;
                }
            }
    if (loss) *loss = L;
    if (dloss) *dloss = dL;
    return VOF_OK;
}

// A recorded switch tape (of one forward run) and its replay.
struct Tape {
    std::vector<uint8_t> bits;
};

template <typename T>
int tape_run(Tape* tp, bool replay, const vof_params* prm, T* F, T* u, T* v, T* w, T* p, int istep0, int nsteps,
             const double* box, double* loss) {
    if (!tp || !prm || !F || !u || !v || !w || !p || nsteps < 0) return VOF_E_INVALID;
    Oracle<T, Taped> o(make_prm(prm, T(0)), 1);
    o.sw.bits = &tp->bits;
    o.sw.replay = replay;
    if (!replay) tp->bits.clear();
    const size_t n = o.N;
    std::copy(F, F + n, o.F.begin());
    std::copy(u, u + n, o.u.begin());
    std::copy(v, v + n, o.v.begin());
    std::copy(w, w + n, o.w.begin());
    std::copy(p, p + n, o.p.begin());
    for (int s = 0; s < nsteps; ++s) o.step(istep0 + s);
    if (replay && (o.sw.overrun || o.sw.pos != tp->bits.size())) return VOF_E_STATE;
    std::copy(o.F.begin(), o.F.end(), F);
    std::copy(o.u.begin(), o.u.end(), u);
    std::copy(o.v.begin(), o.v.end(), v);
    std::copy(o.w.begin(), o.w.end(), w);
    std::copy(o.p.begin(), o.p.end(), p);
    if (loss && box) *loss = box_loss(o, Box{box[0], box[1], box[2], box[3], box[4], box[5]});
    return VOF_OK;
}

}  // namespace

extern "C" {

// dL/d(initial state) and dL/dg of L = sum over the box of F dV after nsteps
// steps from istep0; the forward in FP32 (the CUDA plain path's arithmetic) or
// FP64.  box = {x0, x1, y0, y1, z0, z1} (strict bounds on cell centres).
int oracle_adjoint_f32(const vof_params* prm, const float* F, const float* u, const float* v, const float* w,
                       const float* p, int istep0, int nsteps, const double* box, double* lF, double* lu, double* lv,
                       double* lw, double* lp, double* grad_g, double* loss, int nthreads) {
    return adjoint_run<float>(prm, F, u, v, w, p, istep0, nsteps, box, lF, lu, lv, lw, lp, grad_g, loss, nthreads);
}

int oracle_adjoint_f64(const vof_params* prm, const double* F, const double* u, const double* v, const double* w,
                       const double* p, int istep0, int nsteps, const double* box, double* lF, double* lu,
                       double* lv, double* lw, double* lp, double* grad_g, double* loss, int nthreads) {
    return adjoint_run<double>(prm, F, u, v, w, p, istep0, nsteps, box, lF, lu, lv, lw, lp, grad_g, loss, nthreads);
}

// Directional derivative of the box loss along (dF, du, dv, dw, dp) of the
// initial state and dg of the body force (any may be NULL), by the
// tangent-linear FP64 forward; loss = the FP64 loss itself.
int oracle_tangent_f64(const vof_params* prm, const double* F, const double* u, const double* v, const double* w,
                       const double* p, const double* dF, const double* du, const double* dv, const double* dw,
                       const double* dp, const double* dg, int istep0, int nsteps, const double* box, double* loss,
                       double* dloss, int nthreads) {
    const double* x0[5] = {F, u, v, w, p};
    const double* dx0[5] = {dF, du, dv, dw, dp};
    return tangent_run(prm, x0, dx0, dg, istep0, nsteps, box, loss, dloss, nthreads);
}

// The same with the convergent pressure solve (CG to ||r|| <= tol ||b||, mean
// zero) in every step: the host adjoint of VOF_MODE_MIXED / VOF_MODE_FP64.
int oracle_adjoint_conv_f32(const vof_params* prm, const float* F, const float* u, const float* v, const float* w,
                            const float* p, int istep0, int nsteps, const double* box, double* lF, double* lu,
                            double* lv, double* lw, double* lp, double* grad_g, double* loss, double tol,
                            int nthreads) {
    if (!(tol > 0)) return VOF_E_INVALID;
    return adjoint_run<float>(prm, F, u, v, w, p, istep0, nsteps, box, lF, lu, lv, lw, lp, grad_g, loss, nthreads,
                              tol);
}

int oracle_adjoint_conv_f64(const vof_params* prm, const double* F, const double* u, const double* v,
                            const double* w, const double* p, int istep0, int nsteps, const double* box, double* lF,
                            double* lu, double* lv, double* lw, double* lp, double* grad_g, double* loss, double tol,
                            int nthreads) {
    if (!(tol > 0)) return VOF_E_INVALID;
    return adjoint_run<double>(prm, F, u, v, w, p, istep0, nsteps, box, lF, lu, lv, lw, lp, grad_g, loss, nthreads,
                               tol);
}

void* oracle_tape_new(void) { return new Tape(); }
void oracle_tape_free(void* t) { delete static_cast<Tape*>(t); }
long long oracle_tape_size(void* t) { return t ? (long long)static_cast<Tape*>(t)->bits.size() : -1; }

// A forward run (state updated in place) that records (replay = 0) or replays
// (replay = 1) every switch; loss (optional) = the box loss at the end.
int oracle_tape_run_f64(void* t, int replay, const vof_params* prm, double* F, double* u, double* v, double* w,
                        double* p, int istep0, int nsteps, const double* box, double* loss) {
    return tape_run<double>(static_cast<Tape*>(t), replay != 0, prm, F, u, v, w, p, istep0, nsteps, box, loss);
}

int oracle_tape_run_f32(void* t, int replay, const vof_params* prm, float* F, float* u, float* v, float* w, float* p,
                        int istep0, int nsteps, const double* box, double* loss) {
    return tape_run<float>(static_cast<Tape*>(t), replay != 0, prm, F, u, v, w, p, istep0, nsteps, box, loss);
}

}  // extern "C"
