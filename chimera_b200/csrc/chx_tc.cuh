// chx_tc.cuh -- tcgen05 building blocks shared by the tensor-core kernels of
// libchimera_b200: shared-memory matrix descriptors of the no-swizzle
// K-major layout, mbarriers with bounded waits, MMA completion commits.
#pragma once
#include "chx_common.cuh"

namespace chx {

constexpr uint32_t kTcLBO = 128;                        // core matrices along K (bytes)
constexpr int kTcSpin = 1 << 24;                        // polls of a bounded wait

__device__ __forceinline__ uint32_t tc_smem(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: start address, leading (K) and stride
// (row-group) byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)(kTcLBO >> 4) << 16) |
           ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ bool tc_mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = tc_smem(bar);
    for (int it = 0; it < kTcSpin; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            tc_smem(bar))
        : "memory");
}

}  // namespace chx
