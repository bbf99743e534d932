// tma_host.cu -- host-side tensor-map encoding for the TMA loads (tma.cuh).
// cuTensorMapEncodeTiled is reached through cudaGetDriverEntryPoint, so the
// library needs no link against libcuda.
#include <cudaTypedefs.h>

#include "tma.cuh"

namespace vof {

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

cudaError_t make_tensor_map_3d(CUtensorMap* map, const float* base, int px, int py, int pz, int bx, int by,
                               int bz) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    const cuuint64_t dims[3] = {(cuuint64_t)px, (cuuint64_t)py, (cuuint64_t)pz};
    const cuuint64_t strides[2] = {(cuuint64_t)px * sizeof(float), (cuuint64_t)px * py * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box,
                          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace vof
