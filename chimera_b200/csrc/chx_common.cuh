// chx_common.cuh -- shared device helpers for libchimera_b200 (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <algorithm>
#include <type_traits>
#include "../../include/chimera_b200.h"

namespace chx {

// ------------------------------------------------------------- host errors
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

#define CHX_CHECK_LAUNCH(what)                                      \
    do {                                                            \
        cudaError_t e_ = cudaGetLastError();                        \
        if (e_ != cudaSuccess) return chx::cuda_fail(e_, what);     \
    } while (0)

#define CHX_REQUIRE(cond, ...)                                      \
    do {                                                            \
        if (!(cond)) { chx::set_error(__VA_ARGS__); return CHX_ERR_ARG; } \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int kNumSMs = 148;

// ------------------------------------------------------------ counter RNG
// splitmix64 and its top-53-bit uniform, as the reference's proposal kernel
// defines them (exafs_gpu/kernels.py:352-360): a published mixing function
// (Steele, Lea & Flood 2014) reproduced so that the proposal stream keyed
// (seed, step, replica) is bit-identical.
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ double u01(uint64_t h) {
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

constexpr double kTwoPi = 6.283185307179586;
constexpr double kInvTwoPi = 0.15915494309189535;

// Reduce a phase to [-pi, pi] in FP64 before the FP32 sine: n = rint(x/2pi),
// x - 2 pi n with the product and difference in FP64. |x| stays below a few
// thousand radians here, so the FP64 rounding of 2 pi n is far below FP32's.
__device__ __forceinline__ float reduce_phase(double x) {
    double n = rint(x * kInvTwoPi);
    return (float)fma(-n, kTwoPi, x);
}

template <int NSP>
__device__ __forceinline__ void add_by_species(double (&acc)[NSP], int s, double v) {
#pragma unroll
    for (int q = 0; q < NSP; ++q)
        if (q == s) acc[q] += v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace chx
