// divtest.cu -- test-only library: evaluates the library's device helpers
// (vof_device.cuh) next to CUDA's own operations on caller-supplied operands.
// Built by __graft_entry__.build() into tests/_build/libvof_divtest.so; used
// only by tests/test_division_gpu.py.
#include <cuda_runtime.h>

#include "../../cuda-lbm-ibm-fvm_b200/csrc/vof_device.cuh"

__global__ void k_div(const float* __restrict__ x, const float* __restrict__ d, float* __restrict__ fast,
                      float* __restrict__ ieee, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float rd = __frcp_rn(d[t]);
    fast[t] = vof::div_rn_pre(x[t], d[t], rd);
    ieee[t] = __fdiv_rn(x[t], d[t]);
}

__global__ void k_rcp64(const double* __restrict__ x, double* __restrict__ fast, double* __restrict__ ieee, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    fast[t] = vof::rcp64(x[t]);
    ieee[t] = __drcp_rn(x[t]);
}

// vof::rcp64 next to CUDA's correctly rounded FP64 reciprocal.
extern "C" int rcp64test_run(const double* hx, double* hfast, double* hieee, int n) {
    double *x = nullptr, *f = nullptr, *q = nullptr;
    const size_t b = (size_t)n * sizeof(double);
    int rc = 0;
    if (cudaMalloc(&x, b) || cudaMalloc(&f, b) || cudaMalloc(&q, b)) rc = 1;
    if (!rc && cudaMemcpy(x, hx, b, cudaMemcpyHostToDevice)) rc = 2;
    if (!rc) {
        k_rcp64<<<(n + 255) / 256, 256>>>(x, f, q, n);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = 3;
    }
    if (!rc && (cudaMemcpy(hfast, f, b, cudaMemcpyDeviceToHost) || cudaMemcpy(hieee, q, b, cudaMemcpyDeviceToHost)))
        rc = 4;
    cudaFree(x);
    cudaFree(f);
    cudaFree(q);
    return rc;
}

extern "C" int divtest_run(const float* hx, const float* hd, float* hfast, float* hieee, int n) {
    float *x = nullptr, *d = nullptr, *f = nullptr, *q = nullptr;
    const size_t b = (size_t)n * sizeof(float);
    int rc = 0;
    if (cudaMalloc(&x, b) || cudaMalloc(&d, b) || cudaMalloc(&f, b) || cudaMalloc(&q, b)) rc = 1;
    if (!rc && (cudaMemcpy(x, hx, b, cudaMemcpyHostToDevice) || cudaMemcpy(d, hd, b, cudaMemcpyHostToDevice))) rc = 2;
    if (!rc) {
        k_div<<<(n + 255) / 256, 256>>>(x, d, f, q, n);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = 3;
    }
    if (!rc && (cudaMemcpy(hfast, f, b, cudaMemcpyDeviceToHost) || cudaMemcpy(hieee, q, b, cudaMemcpyDeviceToHost)))
        rc = 4;
    cudaFree(x);
    cudaFree(d);
    cudaFree(f);
    cudaFree(q);
    return rc;
}
