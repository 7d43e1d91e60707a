// chx_mlp.cuh -- one surrogate evaluation by one CTA. The sampler's stage 1
// and chx_mlp_predict run this same function, so their outputs agree bit for
// bit. Weights BF16, activations rounded to BF16 between layers (as the
// training forward does), sums in FP32.
#pragma once
#include <cuda_bf16.h>
#include "chx_common.cuh"

namespace chx {

__device__ __forceinline__ float bf16f(uint16_t h) { return __uint_as_float((uint32_t)h << 16); }

// round to the nearest BF16 (ties to even) and back to FP32
__device__ __forceinline__ float bf16_round(float x) {
    return __bfloat162float(__float2bfloat16_rn(x));
}

// 8 BF16 weights of a 16-byte word, times x, added into acc
__device__ __forceinline__ void fma8(float *acc, uint4 w, float x) {
    const uint32_t u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        acc[2 * j] = fmaf(__uint_as_float(u[j] << 16), x, acc[2 * j]);
        acc[2 * j + 1] = fmaf(__uint_as_float(u[j] & 0xFFFF0000u), x, acc[2 * j + 1]);
    }
}

// Scratch: part (nwarps * H floats) and h (H floats), 16-byte aligned.
// Warp w takes rows w, w + nwarps, ...; lane l < H/8 takes outputs 8l..8l+7
// with one 16-byte load per row; partial sums are reduced over the warps in
// fixed order. Layer 1 rows are the one-hot rows named by codes (1 + 2D
// bytes: the pair row, then the neighbour codes) and, for 0 <= chain <
// nchain, the chain's row. Requires H % 8 == 0, H <= 256 and blockDim.x a
// multiple of 32; every thread of the CTA calls it (it synchronises).
// Returns the network output in every thread.
static __device__ __noinline__ float mlp_eval_cta(const chx_mlp_t &P, const uint8_t *s_codes,
                                                  float lnbeta, int chain, float *part,
                                                  float *h) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int H = P.H, ncg = H >> 3, D2 = 2 * P.D, ns1 = P.nsp + 1;
    const int npt = P.nsp * (P.nsp - 1) / 2;
    const bool col = lane < ncg;
    const int nrow = D2 + ((chain >= 0 && chain < P.nchain) ? 2 : 1);
    float acc[8];
    // ---- layer 1: one W1 row per input site (and the chain's row)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = 0.f;
    if (col) {
        const uint4 *W = (const uint4 *)P.W1;
#pragma unroll 4
        for (int k = warp; k < nrow; k += nw) {
            const int row = k == 0 ? (int)s_codes[0]
                                   : (k <= D2 ? npt + (k - 1) * ns1 + (int)s_codes[k]
                                              : npt + D2 * ns1 + chain);
            fma8(acc, __ldg(&W[(long)row * ncg + lane]), 1.f);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) part[warp * H + 8 * lane + j] = acc[j];
    }
    __syncthreads();
    const float f = (lnbeta - P.feat_shift) * P.feat_scale;
    for (int o = tid; o < H; o += blockDim.x) {
        float s = fmaf(f, bf16f(P.W1[(long)P.nin * H + o]), P.b1[o]);
        for (int w = 0; w < nw; ++w) s += part[w * H + o];
        h[o] = bf16_round(fmaxf(s, 0.f));
    }
    __syncthreads();
    // ---- layers 2 and 3: dense H x H
#pragma unroll 1
    for (int layer = 0; layer < 2; ++layer) {
        const uint4 *W = (const uint4 *)(layer == 0 ? P.W2 : P.W3);
        const float *bias = layer == 0 ? P.b2 : P.b3;
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] = 0.f;
        if (col) {
#pragma unroll 8
            for (int i = warp; i < H; i += nw) fma8(acc, __ldg(&W[(long)i * ncg + lane]), h[i]);
        }
        __syncthreads();   // every h[i] read before it is overwritten
        if (col) {
#pragma unroll
            for (int j = 0; j < 8; ++j) part[warp * H + 8 * lane + j] = acc[j];
        }
        __syncthreads();
        for (int o = tid; o < H; o += blockDim.x) {
            float s = bias[o];
            for (int w = 0; w < nw; ++w) s += part[w * H + o];
            h[o] = bf16_round(fmaxf(s, 0.f));
        }
        __syncthreads();
    }
    // ---- output: warp 0 sums h . w4 in fixed lane order, broadcast through part
    if (warp == 0) {
        float s = 0.f;
        for (int i = lane; i < H; i += 32) s = fmaf(h[i], bf16f(P.w4[i]), s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) part[0] = s + P.b4[0];
    }
    __syncthreads();
    const float y = part[0];
    __syncthreads();
    return y;
}

// Row of the unordered species pair {p, q}, p != q, among nsp(nsp-1)/2.
__device__ __host__ __forceinline__ int pair_row(int p, int q, int nsp) {
    int lo = p < q ? p : q, hi = p < q ? q : p;
    return lo * nsp - lo * (lo + 1) / 2 + (hi - lo - 1);
}

}  // namespace chx
