// ref_harness.cu -- drives the reference's own kernels on caller-supplied state.
//
// TEST INFRASTRUCTURE ONLY (used by tests/, tests/golden/gen_golden.py and
// bench.py --impl reference).  Built by oracle/Makefile, which puts the
// reference source directory on the include path and renames its main():
//     nvcc ... -I<reference dir> -Dmain=voftrial1_main ref_harness.cu
// so the translation unit below is the reference's voftrial1.cu unmodified
// plus this file's extern "C" entry points.  Outputs go to oracle/_ref/ only.
//
// The entry points fill cpar_host from a vof_params (which mirrors Params,
// voftrial1.cu:27-41), allocate DeviceFields with the reference's alloc_field,
// upload host state in the reference layout and run the time-loop body of
// voftrial1.cu:1364-1401 with the reference's launch shapes
// (voftrial1.cu:1340-1356).  The Jacobi sweep count comes from
// vof_params::jacobi_iters (the reference hardcodes 10, voftrial1.cu:1371).
#include "voftrial1.cu"

#include "../include/vof.h"

namespace {

void load_params(const vof_params* p) {
    cpar_host.nx = p->nx;
    cpar_host.ny = p->ny;
    cpar_host.nz = p->nz;
    cpar_host.imin = p->imin;
    cpar_host.imax = p->imax;
    cpar_host.jmin = p->jmin;
    cpar_host.jmax = p->jmax;
    cpar_host.kmin = p->kmin;
    cpar_host.kmax = p->kmax;
    cpar_host.Lx = p->Lx;
    cpar_host.Ly = p->Ly;
    cpar_host.Lz = p->Lz;
    cpar_host.rho_l = p->rho_l;
    cpar_host.rho_g = p->rho_g;
    cpar_host.nu_l = p->nu_l;
    cpar_host.nu_g = p->nu_g;
    cpar_host.sigma = p->sigma;
    cpar_host.gx = p->gx;
    cpar_host.gy = p->gy;
    cpar_host.gz = p->gz;
    cpar_host.dt = p->dt;
    cpar_host.dx = p->dx;
    cpar_host.dy = p->dy;
    cpar_host.dz = p->dz;
    cpar_host.dxi = p->dxi;
    cpar_host.dyi = p->dyi;
    cpar_host.dzi = p->dzi;
    cpar_host.nTot = p->nTot;
    CHECK_CUDA(cudaMemcpyToSymbol(cpar, &cpar_host, sizeof(Params)));
}

struct Launch {
    dim3 block3d, gridXYZ, gridU, gridV, gridW;
    int threads1d, blocks1d;
};

Launch shapes(const vof_params* p) {
    Launch L;
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    L.block3d = dim3(8, 8, 4);
    L.gridXYZ = dim3((nx + 7) / 8, (ny + 7) / 8, (nz + 3) / 4);
    L.gridU = dim3((std::max(nx - 1, 1) + 7) / 8, (ny + 7) / 8, (nz + 3) / 4);
    L.gridV = dim3((nx + 7) / 8, (std::max(ny - 1, 1) + 7) / 8, (nz + 3) / 4);
    L.gridW = dim3((nx + 7) / 8, (ny + 7) / 8, (std::max(nz - 1, 1) + 3) / 4);
    L.threads1d = 256;
    L.blocks1d = (p->nTot + 255) / 256;
    return L;
}

void alloc_all(DeviceFields& d, size_t bytes) {
    alloc_field(&d.F, bytes);
    alloc_field(&d.Ftd, bytes);
    alloc_field(&d.ax, bytes);
    alloc_field(&d.ay, bytes);
    alloc_field(&d.az, bytes);
    alloc_field(&d.cx, bytes);
    alloc_field(&d.cy, bytes);
    alloc_field(&d.cz, bytes);
    alloc_field(&d.rp, bytes);
    alloc_field(&d.rm, bytes);
    alloc_field(&d.u, bytes);
    alloc_field(&d.v, bytes);
    alloc_field(&d.w, bytes);
    alloc_field(&d.u_star, bytes);
    alloc_field(&d.v_star, bytes);
    alloc_field(&d.w_star, bytes);
    alloc_field(&d.p, bytes);
    alloc_field(&d.pt, bytes);
    alloc_field(&d.rho, bytes);
    alloc_field(&d.nu, bytes);
}

// The body of the reference's time loop for one istep.
void one_step(DeviceFields& d, const Launch& L, int istep, int jacobi_iters) {
    cal_nu_rho_kernel<<<L.blocks1d, L.threads1d>>>(d.F, d.rho, d.nu);
    advect_u_kernel<<<L.gridU, L.block3d>>>(d.u, d.v, d.w, d.rho, d.nu, d.u_star);
    advect_v_kernel<<<L.gridV, L.block3d>>>(d.u, d.v, d.w, d.rho, d.nu, d.v_star);
    advect_w_kernel<<<L.gridW, L.block3d>>>(d.u, d.v, d.w, d.rho, d.nu, d.w_star);
    CHECK_CUDA(cudaPeekAtLastError());
    for (int it = 0; it < jacobi_iters; ++it) {
        solve_p_jacobi_kernel<<<L.gridXYZ, L.block3d>>>(d.u_star, d.v_star, d.w_star, d.rho, d.p, d.pt);
        CHECK_CUDA(cudaPeekAtLastError());
        std::swap(d.p, d.pt);
    }
    update_u_kernel<<<L.gridU, L.block3d>>>(d.rho, d.u_star, d.p, d.u);
    update_v_kernel<<<L.gridV, L.block3d>>>(d.rho, d.v_star, d.p, d.v);
    update_w_kernel<<<L.gridW, L.block3d>>>(d.rho, d.w_star, d.p, d.w);
    CHECK_CUDA(cudaPeekAtLastError());
    apply_bc_velocity(d.u, d.v, d.w);
    if (istep % 3 == 0) {
        run_fct_x(d.F, d.Ftd, d.u, d.ax, d.ay, d.cx, d.cy, d.rp, d.rm);
        run_fct_y(d.F, d.Ftd, d.v, d.ax, d.ay, d.cx, d.cy, d.rp, d.rm);
        run_fct_z(d.F, d.Ftd, d.w, d.az, d.cz, d.rp, d.rm);
    } else if (istep % 3 == 1) {
        run_fct_y(d.F, d.Ftd, d.v, d.ax, d.ay, d.cx, d.cy, d.rp, d.rm);
        run_fct_z(d.F, d.Ftd, d.w, d.az, d.cz, d.rp, d.rm);
        run_fct_x(d.F, d.Ftd, d.u, d.ax, d.ay, d.cx, d.cy, d.rp, d.rm);
    } else {
        run_fct_z(d.F, d.Ftd, d.w, d.az, d.cz, d.rp, d.rm);
        run_fct_x(d.F, d.Ftd, d.u, d.ax, d.ay, d.cx, d.cy, d.rp, d.rm);
        run_fct_y(d.F, d.Ftd, d.v, d.ax, d.ay, d.cx, d.cy, d.rp, d.rm);
    }
    post_process_f_kernel<<<L.blocks1d, L.threads1d>>>(d.F);
    CHECK_CUDA(cudaPeekAtLastError());
    apply_bc_F(d.F);
}

void upload(DeviceFields& d, size_t bytes, const float* F, const float* u, const float* v, const float* w,
            const float* p) {
    CHECK_CUDA(cudaMemcpy(d.F, F, bytes, cudaMemcpyHostToDevice));
    CHECK_CUDA(cudaMemcpy(d.u, u, bytes, cudaMemcpyHostToDevice));
    CHECK_CUDA(cudaMemcpy(d.v, v, bytes, cudaMemcpyHostToDevice));
    CHECK_CUDA(cudaMemcpy(d.w, w, bytes, cudaMemcpyHostToDevice));
    CHECK_CUDA(cudaMemcpy(d.p, p, bytes, cudaMemcpyHostToDevice));
}

}  // namespace

extern "C" {

// Run nsteps reference steps (istep0, istep0+1, ...) on the host state given
// in the reference layout; the state arrays are overwritten with the result.
// us/vs/ws (may be NULL) receive the last step's u_star/v_star/w_star.
int ref_run(const vof_params* prm, float* F, float* u, float* v, float* w, float* p, int istep0, int nsteps,
            float* us, float* vs, float* ws) {
    if (!prm || !F || !u || !v || !w || !p || nsteps < 0) return VOF_E_INVALID;
    load_params(prm);
    const size_t bytes = (size_t)prm->nTot * sizeof(float);
    DeviceFields d;
    alloc_all(d, bytes);
    upload(d, bytes, F, u, v, w, p);
    const Launch L = shapes(prm);
    for (int s = 0; s < nsteps; ++s) one_step(d, L, istep0 + s, prm->jacobi_iters);
    CHECK_CUDA(cudaDeviceSynchronize());
    CHECK_CUDA(cudaMemcpy(F, d.F, bytes, cudaMemcpyDeviceToHost));
    CHECK_CUDA(cudaMemcpy(u, d.u, bytes, cudaMemcpyDeviceToHost));
    CHECK_CUDA(cudaMemcpy(v, d.v, bytes, cudaMemcpyDeviceToHost));
    CHECK_CUDA(cudaMemcpy(w, d.w, bytes, cudaMemcpyDeviceToHost));
    CHECK_CUDA(cudaMemcpy(p, d.p, bytes, cudaMemcpyDeviceToHost));
    if (us) CHECK_CUDA(cudaMemcpy(us, d.u_star, bytes, cudaMemcpyDeviceToHost));
    if (vs) CHECK_CUDA(cudaMemcpy(vs, d.v_star, bytes, cudaMemcpyDeviceToHost));
    if (ws) CHECK_CUDA(cudaMemcpy(ws, d.w_star, bytes, cudaMemcpyDeviceToHost));
    free_all(d);
    return VOF_OK;
}

// Time the reference loop body: `warmup` untimed steps, then `nsteps` steps
// bracketed by CUDA events on the legacy default stream (the stream the
// reference launches on).  *ms_out = elapsed milliseconds of the timed steps.
// If F_out is not NULL it receives F after the timed steps.
int ref_time(const vof_params* prm, const float* F, const float* u, const float* v, const float* w,
             const float* p, int istep0, int warmup, int nsteps, double* ms_out, float* F_out) {
    if (!prm || !F || !u || !v || !w || !p || !ms_out || nsteps < 0 || warmup < 0) return VOF_E_INVALID;
    load_params(prm);
    const size_t bytes = (size_t)prm->nTot * sizeof(float);
    DeviceFields d;
    alloc_all(d, bytes);
    upload(d, bytes, F, u, v, w, p);
    const Launch L = shapes(prm);
    int istep = istep0;
    for (int s = 0; s < warmup; ++s) one_step(d, L, istep++, prm->jacobi_iters);
    cudaEvent_t e0, e1;
    CHECK_CUDA(cudaEventCreate(&e0));
    CHECK_CUDA(cudaEventCreate(&e1));
    CHECK_CUDA(cudaDeviceSynchronize());
    CHECK_CUDA(cudaEventRecord(e0, 0));
    for (int s = 0; s < nsteps; ++s) one_step(d, L, istep++, prm->jacobi_iters);
    CHECK_CUDA(cudaEventRecord(e1, 0));
    CHECK_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *ms_out = ms;
    if (F_out) CHECK_CUDA(cudaMemcpy(F_out, d.F, bytes, cudaMemcpyDeviceToHost));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    free_all(d);
    return VOF_OK;
}

// Kernel launches the reference enqueues per step.
int ref_kernels_per_step(int jacobi_iters) { return 1 + 3 + jacobi_iters + 3 + 3 + 3 * 4 + 1 + 3; }

// The reference's initial condition: set_init_F_kernel with its launch shape
// and one apply_bc_F (voftrial1.cu:1328-1337); F_out gets nTot floats.
int ref_initial_F(const vof_params* prm, int ic, float* F_out) {
    if (!prm || !F_out) return VOF_E_INVALID;
    load_params(prm);
    const size_t bytes = (size_t)prm->nTot * sizeof(float);
    float* F = nullptr;
    alloc_field(&F, bytes);
    const dim3 blockInit(8, 8, 4);
    const dim3 gridInit((prm->nx + 2 + blockInit.x - 1) / blockInit.x, (prm->ny + 2 + blockInit.y - 1) / blockInit.y,
                        (prm->nz + 2 + blockInit.z - 1) / blockInit.z);
    set_init_F_kernel<<<gridInit, blockInit>>>(F, ic);
    CHECK_CUDA(cudaPeekAtLastError());
    apply_bc_F(F);
    CHECK_CUDA(cudaDeviceSynchronize());
    CHECK_CUDA(cudaMemcpy(F_out, F, bytes, cudaMemcpyDeviceToHost));
    cudaFree(F);
    return VOF_OK;
}

// The reference's apply_bc (voftrial1.cu:943-956, set_bc_{j,i,k}_kernel) on
// six host fields in the reference layout, updated in place.
int ref_apply_bc(const vof_params* prm, float* u, float* v, float* w, float* F, float* p, float* rho) {
    if (!prm || !u || !v || !w || !F || !p || !rho) return VOF_E_INVALID;
    load_params(prm);
    const size_t bytes = (size_t)prm->nTot * sizeof(float);
    float* host[6] = {u, v, w, F, p, rho};
    float* dev[6] = {};
    for (int q = 0; q < 6; ++q) {
        alloc_field(&dev[q], bytes);
        CHECK_CUDA(cudaMemcpy(dev[q], host[q], bytes, cudaMemcpyHostToDevice));
    }
    apply_bc(dev[0], dev[1], dev[2], dev[3], dev[4], dev[5]);
    CHECK_CUDA(cudaDeviceSynchronize());
    for (int q = 0; q < 6; ++q) {
        CHECK_CUDA(cudaMemcpy(host[q], dev[q], bytes, cudaMemcpyDeviceToHost));
        cudaFree(dev[q]);
    }
    return VOF_OK;
}

// The reference's dump writer (write_legacy_vtk, voftrial1.cu:907-941) on a
// host field of nxTot * nyTot * nzTot floats; host code only, no GPU needed.
int ref_write_vtk(const char* path, const float* field, int nxTot, int nyTot, int nzTot) {
    if (!path || !field || nxTot < 2 || nyTot < 2 || nzTot < 2) return VOF_E_INVALID;
    const std::vector<float> f(field, field + (size_t)nxTot * nyTot * nzTot);
    write_legacy_vtk(path, f, nxTot, nyTot, nzTot);
    return VOF_OK;
}

}  // extern "C"
