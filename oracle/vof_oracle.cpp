// vof_oracle.cpp -- CPU restatement of the voftrial1.cu time step (the
// forward oracle; the step itself is in oracle_core.h).
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle of the CUDA step in
// cuda-lbm-ibm-fvm_b200/csrc; it is loaded only by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product
// never links or calls it.
#include "oracle_core.h"

namespace {
using namespace vofo;

template <typename T>
int run(const vof_params* prm, T* F, T* u, T* v, T* w, T* p, int istep0, int nsteps, T* us_out,
        T* vs_out, T* ws_out, T* rhs_out, int nthreads, double conv_tol = 0.0) {
    if (!prm || !F || !u || !v || !w || !p || nsteps < 0) return VOF_E_INVALID;
    if (prm->nx < 1 || prm->ny < 1 || prm->nz < 1) return VOF_E_SIZE;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    Oracle<T> o(make_prm(prm, T(0)), nthreads);
    o.conv_tol = conv_tol;
    const size_t n = o.N;
    std::copy(F, F + n, o.F.begin());
    std::copy(u, u + n, o.u.begin());
    std::copy(v, v + n, o.v.begin());
    std::copy(w, w + n, o.w.begin());
    std::copy(p, p + n, o.p.begin());
    for (int s = 0; s < nsteps; ++s) o.step(istep0 + s);
    std::copy(o.F.begin(), o.F.end(), F);
    std::copy(o.u.begin(), o.u.end(), u);
    std::copy(o.v.begin(), o.v.end(), v);
    std::copy(o.w.begin(), o.w.end(), w);
    std::copy(o.p.begin(), o.p.end(), p);
    if (us_out) std::copy(o.us.begin(), o.us.end(), us_out);
    if (vs_out) std::copy(o.vs.begin(), o.vs.end(), vs_out);
    if (ws_out) std::copy(o.ws.begin(), o.ws.end(), ws_out);
    if (rhs_out) {
        std::vector<T> r;
        o.rhs_field(r);
        std::copy(r.begin(), r.end(), rhs_out);
    }
    return VOF_OK;
}

}  // namespace

extern "C" {

// Run nsteps reference steps starting at istep0 on the given state (reference
// layout, nTot values each, updated in place).  Optional outputs (may be NULL):
// the last step's u*, v*, w* and rho/dt*div(u*).
int oracle_run_f32(const vof_params* prm, float* F, float* u, float* v, float* w, float* p, int istep0,
                   int nsteps, float* us, float* vs, float* ws, float* rhs, int nthreads) {
    return run<float>(prm, F, u, v, w, p, istep0, nsteps, us, vs, ws, rhs, nthreads);
}

int oracle_run_f64(const vof_params* prm, double* F, double* u, double* v, double* w, double* p, int istep0,
                   int nsteps, double* us, double* vs, double* ws, double* rhs, int nthreads) {
    return run<double>(prm, F, u, v, w, p, istep0, nsteps, us, vs, ws, rhs, nthreads);
}

// FP64 steps with the convergent pressure solve (CG to ||r|| <= tol ||b||,
// gauge mean(p) = 0) in place of the Jacobi sweeps: the FP64 oracle of
// VOF_MODE_MIXED / VOF_MODE_FP64.
int oracle_run_conv_f64(const vof_params* prm, double* F, double* u, double* v, double* w, double* p, int istep0,
                        int nsteps, double tol, int nthreads) {
    if (!(tol > 0)) return VOF_E_INVALID;
    return run<double>(prm, F, u, v, w, p, istep0, nsteps, nullptr, nullptr, nullptr, nullptr, nthreads, tol);
}

// The reference's apply_bc (voftrial1.cu:943-956) on six host fields in the
// reference layout, updated in place.
int oracle_apply_bc_f32(const vof_params* prm, float* u, float* v, float* w, float* F, float* p, float* rho) {
    if (!prm || !u || !v || !w || !F || !p || !rho) return VOF_E_INVALID;
    if (prm->nx < 1 || prm->ny < 1 || prm->nz < 1) return VOF_E_SIZE;
    Oracle<float> o(make_prm(prm, 0.0f), 1);
    float* fields[6] = {u, v, w, F, p, rho};
    std::vector<float>* mine[6] = {&o.u, &o.v, &o.w, &o.F, &o.p, &o.rho};
    for (int q = 0; q < 6; ++q) std::copy(fields[q], fields[q] + o.N, mine[q]->begin());
    o.bc_all();
    for (int q = 0; q < 6; ++q) std::copy(mine[q]->begin(), mine[q]->end(), fields[q]);
    return VOF_OK;
}

// clamp01f of the reference on one value, in float and in double.
float oracle_clamp01f(float v) { return clamp01<float>(v); }
double oracle_clamp01d(double v) { return clamp01<double>(v); }

int oracle_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
