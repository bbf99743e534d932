// tma.cuh -- Tensor Memory Accelerator (cp.async.bulk.tensor) loads and
// mbarrier helpers for sm_100a, in inline PTX, plus host-side tensor-map
// encoding through the driver entry point (no link against libcuda).
//
// Only plain (non-multicast) tiled and untiled bulk loads of this GPU's own
// memory are used.
// Every wait is bounded: a wait that runs out of iterations reports failure
// and the kernel records it in a device status word instead of hanging.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace vof {

// Status word codes written by kernels (0 = fine).
enum : int { DEV_OK = 0, DEV_TMA_TIMEOUT = 1 };

// Spin limit of one mbarrier wait (each try_wait itself blocks for a
// hardware-defined interval); far above any legitimate plane latency.
constexpr uint32_t MBAR_SPIN_LIMIT = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make mbarrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Wait for phase `parity` of the barrier to complete, at most `limit` tries;
// false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = MBAR_SPIN_LIMIT) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// One arrival on the barrier (no transaction bytes).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Untiled bulk copy of `bytes` bytes (a multiple of 16; both addresses
// 16-byte aligned) from this GPU's global memory into shared memory,
// completing on `bar` (complete_tx).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// 3D tiled TMA load of one box at element coordinates (x, y, z) into shared
// memory, completing on `bar` (complete_tx).  x * 4 bytes must be a multiple
// of 16 for float tensors.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Host: encode a 3D float32 tensor map over a padded field (dims px, py, pz
// elements, x fastest) with box (bx, by, bz); out-of-bounds reads give 0.
cudaError_t make_tensor_map_3d(CUtensorMap* map, const float* base, int px, int py, int pz, int bx, int by,
                               int bz);

}  // namespace vof
