// apply_bc.cu -- the reference's apply_bc (voftrial1.cu:943-956) as one
// in-place launch.
//
// The reference runs set_bc_j_kernel, set_bc_i_kernel and set_bc_k_kernel
// (voftrial1.cu:105-228) one after the other.  Followed through the three
// passes, each boundary value has a closed form in the fields as they were
// before the call.  With ci, cj, ck the indices clamped to the interior
// (0 -> 1, n+1 -> n):
//   F, p, rho   every ghost cell (edges and corners included) takes
//               X[ci, cj, ck];
//   u           0 on the faces i = 1 and i = nx+1 (all j, k); elsewhere on
//               the shell u[i, cj, ck] (i itself is not clamped);
//   v           0 on j = 1 and j = ny+1; elsewhere on the shell v[ci, j, ck];
//   w           0 on k = 1 and k = nz+1; elsewhere on the shell w[ci, cj, k].
// Every cell read in these formulas lies where the map leaves the value
// unchanged, so one launch over the shell and the three wall-normal faces,
// in any thread order, gives the result of the three passes.  A cell whose
// source is the cell itself is not written.
//
// The grid is the reference layout (px = nx+2) or the padded one (px a
// multiple of 32): cell (i, j, k) at k*plane + j*px + i.
#include "apply_bc.h"

namespace vof {
namespace {

constexpr int BC_THREADS = 256;

struct BcGrid {
    int nx, ny, nz;
    size_t px, plane;
};

__device__ __forceinline__ size_t at(const BcGrid& g, int i, int j, int k) {
    return (size_t)k * g.plane + (size_t)j * g.px + (size_t)i;
}

__device__ __forceinline__ int clamp_in(int v, int n) { return v < 1 ? 1 : (v > n ? n : v); }

// One cell of the ghost shell: its final value in every field given.
__device__ __forceinline__ void shell_cell(const BcGrid& g, const BcFields& f, int i, int j, int k) {
    const int ci = clamp_in(i, g.nx), cj = clamp_in(j, g.ny), ck = clamp_in(k, g.nz);
    const size_t c = at(g, i, j, k);
    const size_t s = at(g, ci, cj, ck);
    if (f.F) f.F[c] = f.F[s];
    if (f.p) f.p[c] = f.p[s];
    if (f.rho) f.rho[c] = f.rho[s];
    if (f.u) {
        if (i == 1 || i == g.nx + 1) {
            f.u[c] = 0.0f;
        } else {
            const size_t su = at(g, i, cj, ck);
            if (su != c) f.u[c] = f.u[su];
        }
    }
    if (f.v) {
        if (j == 1 || j == g.ny + 1) {
            f.v[c] = 0.0f;
        } else {
            const size_t sv = at(g, ci, j, ck);
            if (sv != c) f.v[c] = f.v[sv];
        }
    }
    if (f.w) {
        if (k == 1 || k == g.nz + 1) {
            f.w[c] = 0.0f;
        } else {
            const size_t sw = at(g, ci, cj, k);
            if (sw != c) f.w[c] = f.w[sw];
        }
    }
}

// Work items, in order: the two k faces (all i, j), the two j faces (all i,
// interior k), the two i faces (interior j, k), then u on i = 1, v on j = 1
// and w on k = 1 over the interior of each face.  x runs fastest where the
// face allows it.
__global__ void __launch_bounds__(BC_THREADS) k_apply_bc(BcGrid g, BcFields f) {
    const long long ex = g.nx + 2, ey = g.ny + 2;
    const long long nA = 2 * ex * ey;
    const long long nB = 2 * ex * g.nz;
    const long long nC = 2 * (long long)g.ny * g.nz;
    const long long nU = (long long)g.ny * g.nz;
    const long long nV = (long long)g.nx * g.nz;
    const long long nW = (long long)g.nx * g.ny;
    const long long total = nA + nB + nC + nU + nV + nW;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        long long r = t;
        if (r < nA) {
            const long long face = r / (ex * ey), q = r % (ex * ey);
            shell_cell(g, f, (int)(q % ex), (int)(q / ex), face ? g.nz + 1 : 0);
            continue;
        }
        r -= nA;
        if (r < nB) {
            const long long face = r / (ex * g.nz), q = r % (ex * g.nz);
            shell_cell(g, f, (int)(q % ex), face ? g.ny + 1 : 0, 1 + (int)(q / ex));
            continue;
        }
        r -= nB;
        if (r < nC) {
            const long long face = r / nU, q = r % nU;
            shell_cell(g, f, face ? g.nx + 1 : 0, 1 + (int)(q % g.ny), 1 + (int)(q / g.ny));
            continue;
        }
        r -= nC;
        if (r < nU) {
            if (f.u) f.u[at(g, 1, 1 + (int)(r % g.ny), 1 + (int)(r / g.ny))] = 0.0f;
            continue;
        }
        r -= nU;
        if (r < nV) {
            if (f.v) f.v[at(g, 1 + (int)(r % g.nx), 1, 1 + (int)(r / g.nx))] = 0.0f;
            continue;
        }
        r -= nV;
        if (f.w) f.w[at(g, 1 + (int)(r % g.nx), 1 + (int)(r / g.nx), 1)] = 0.0f;
    }
}

}  // namespace

cudaError_t apply_bc_launch(int nx, int ny, int nz, int px, const BcFields& f, cudaStream_t s) {
    if (nx < 1 || ny < 1 || nz < 1 || px < nx + 2) return cudaErrorInvalidValue;
    BcGrid g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.px = (size_t)px;
    g.plane = (size_t)px * (size_t)(ny + 2);
    const long long ex = nx + 2, ey = ny + 2;
    const long long total = 2 * ex * ey + 2 * ex * nz + 2LL * ny * nz + (long long)ny * nz + (long long)nx * nz +
                            (long long)nx * ny;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = (total + BC_THREADS - 1) / BC_THREADS;
    const int blocks = (int)(want < 8LL * sms ? want : 8LL * sms);
    k_apply_bc<<<blocks, BC_THREADS, 0, s>>>(g, f);
    return cudaGetLastError();
}

}  // namespace vof
