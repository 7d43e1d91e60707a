// chx_mlp.cu -- the swap surrogate's batch kernels: inference (the same
// per-CTA code the sampler runs), training forward + loss + gradient, Adam.
//
// Training works on a batch of B logged swaps. The two dense layers
// (B x H x H) run on the tcgen05 tensor cores through one strided BF16 GEMM
// (FP32 accumulation in tensor memory) that serves the forward (H W), the
// weight gradients (H^T dZ) and the input gradients (dZ W^T). Layer 1 is a
// gather-sum of W1 rows (its input is one-hot), and its weight gradient a
// per-site scatter done as one CTA per input site with no atomics. Every
// reduction runs in a fixed order, so a gradient is reproducible bit for bit.
// Rounding: weights BF16; activations and the back-propagated dZ rounded to
// BF16 before they enter a GEMM; everything else FP32.
#include "chx_mlp.cuh"
#include "chx_tc.cuh"

namespace chx {

static inline int64_t mlp_nin(int nsp, int D, int nchain) {
    return (int64_t)nsp * (nsp - 1) / 2 + 2LL * D * (nsp + 1) + nchain;
}

// ---------------------------------------------------------------- GEMM
// C[m][n] = sum_k A(m,k) B(k,n) (+ bias[n]); A(m,k) = A[m*sam + k*sak],
// B(k,n) = B[k*sbk + n*sbn] (BF16 bit patterns); C FP32 with row stride ldc;
// with Cb, also BF16(relu(C)) (relu != 0) or BF16(C) into Cb (row stride ldc).
//
// On the tcgen05 tensor cores: one CTA (4 warps) per 128 x 128 tile of C,
// the FP32 accumulator in 128 columns of tensor memory. K goes in chunks of
// 32: all threads stage the chunk's A rows and B columns (any strides, so
// plain loads) into two 8 KB tiles in the no-swizzle K-major core-matrix
// layout (8 x 16-byte core matrices, 128 B apart along K, 512 B per row
// group), then one thread issues two 128 x 128 x 16 BF16 MMAs (kind::f16)
// and commits them to the chunk buffer's mbarrier; two buffers, so the
// staging of chunk c + 1 overlaps the MMAs of chunk c. The epilogue warp w
// reads accumulator lanes 32w..32w+31 (one row each) with tcgen05.ld. Every
// wait is bounded; a wait that runs out makes the tile's outputs NaN after
// the MMAs the CTA issued have completed.
constexpr int kGm = 128, kGn = 128, kGk = 32;
constexpr uint32_t kGsbo = (kGk * 2 / 16) * 128;          // row-group stride of a tile
constexpr uint32_t kGtile = kGm * kGk * 2;                 // one 128 x 32 BF16 tile
constexpr uint32_t kGidesc = (1u << 4) | (1u << 7) | (1u << 10) |
                             ((uint32_t)(kGn >> 3) << 17) | ((uint32_t)(kGm >> 4) << 24);
// two buffers of two tiles and alignment slack, rounded up so that at most
// four CTAs (4 x 128 tensor-memory columns of 512) share an SM
constexpr size_t kGsmem = 57 * 1024;
static_assert(4 * kGtile + 1024 <= kGsmem && 5 * (kGsmem + 1024) > 228 * 1024,
              "GEMM shared memory must hold the buffers and cap the CTAs per SM at four");

// byte offset of element (r, k) in a 128 x 32 BF16 tile
__device__ __forceinline__ uint32_t g_off(int r, int k) {
    return (uint32_t)((r >> 3) * kGsbo + (k >> 3) * kTcLBO + (r & 7) * 16 + (k & 7) * 2);
}

// Stage one 128 x 32 chunk of an operand X(r, k) = X[r*sr + k*sk] (rows
// r0.., K columns k0..) into the core-matrix tile, zero past R and K. mode 1:
// k contiguous (sk == 1), a 16-byte load per 8 k of one row; mode 2: rows
// contiguous (sr == 1), a 16-byte load per 8 rows of one k, scattered into
// the 8 rows' core matrices; mode 0: one element at a time. The vector modes
// need the base 16-byte aligned and the other stride a multiple of 8.
__device__ __forceinline__ void g_stage(uint8_t *tile, const uint16_t *__restrict__ X, long sr,
                                        long sk, int r0, int R, int k0, int K, int mode) {
    const int tid = threadIdx.x;
    if (mode == 1) {
        for (int q = tid; q < kGm * (kGk / 8); q += blockDim.x) {
            const int r = q >> 2, kg = (q & 3) * 8, gr = r0 + r, gk = k0 + kg;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (gr < R) {
                if (gk + 8 <= K) {
                    v = __ldg((const uint4 *)(X + gr * sr + gk));
                } else {
                    __align__(16) uint16_t e[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) e[j] = gk + j < K ? X[gr * sr + gk + j] : (uint16_t)0;
                    v = *(const uint4 *)e;
                }
            }
            *(uint4 *)(tile + g_off(r, kg)) = v;
        }
    } else if (mode == 2) {
        for (int q = tid; q < kGk * (kGm / 8); q += blockDim.x) {
            const int k = q >> 4, rg = (q & 15) * 8, gr = r0 + rg, gk = k0 + k;
            __align__(16) uint16_t e[8];
            if (gk < K && gr + 8 <= R) {
                *(uint4 *)e = __ldg((const uint4 *)(X + (long)gk * sk + gr));
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    e[j] = (gk < K && gr + j < R) ? X[(long)gk * sk + gr + j] : (uint16_t)0;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) *(uint16_t *)(tile + g_off(rg + j, k)) = e[j];
        }
    } else {
        for (int q = tid; q < kGm * (kGk / 8); q += blockDim.x) {
            const int r = q >> 2, kg = (q & 3) * 8, gr = r0 + r, gk = k0 + kg;
            __align__(16) uint16_t e[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
                e[j] = (gr < R && gk + j < K) ? X[gr * sr + (long)(gk + j) * sk] : (uint16_t)0;
            *(uint4 *)(tile + g_off(r, kg)) = *(const uint4 *)e;
        }
    }
}

__device__ __forceinline__ void g_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
            tmem),
        "l"(da), "l"(db), "r"(kGidesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__global__ void __launch_bounds__(128) k_gemm_tc(const uint16_t *__restrict__ A, long sam,
                                                 long sak, const uint16_t *__restrict__ B,
                                                 long sbk, long sbn, float *__restrict__ C,
                                                 long ldc, uint16_t *__restrict__ Cb,
                                                 const float *__restrict__ bias, int M, int N,
                                                 int K, int relu, int kslice) {
    extern __shared__ uint8_t g_raw[];
    __shared__ __align__(8) uint64_t buf_bar[2], done_bar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    uint8_t *sm = (uint8_t *)(((uintptr_t)g_raw + 1023) & ~(uintptr_t)1023);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * kGm, n0 = blockIdx.x * kGn;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         tc_smem(&s_tmem)),
                     "r"(kGn)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        tc_mbar_init(&buf_bar[0], 1);
        tc_mbar_init(&buf_bar[1], 1);
        tc_mbar_init(&done_bar, 1);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    // split K: block z takes K range [z kslice, (z + 1) kslice) and writes its
    // partial product to the z-th M x ldc slab of C
    const int kbeg = blockIdx.z * kslice, kend = min(K, kbeg + kslice);
    const int nkc = kend > kbeg ? (kend - kbeg + kGk - 1) / kGk : 0;
    C += (long)blockIdx.z * M * ldc;
    auto mode_of = [](const uint16_t *X, long sr, long sk) {
        if (((uintptr_t)X & 15) != 0) return 0;
        if (sk == 1 && sr % 8 == 0) return 1;
        if (sr == 1 && sk % 8 == 0) return 2;
        return 0;
    };
    const int va_mode = mode_of(A, sam, sak), vb_mode = mode_of(B, sbn, sbk);
    for (int kc = 0; kc < nkc; ++kc) {
        const int b = kc & 1;
        uint8_t *sa = sm + (size_t)b * 2 * kGtile, *sb = sa + kGtile;
        // the buffer's previous chunk (kc - 2) has been read by its MMAs
        if (kc >= 2 && !tc_mbar_wait(&buf_bar[b], (uint32_t)((kc / 2 - 1) & 1))) s_fail = 1;
        __syncthreads();
        if (s_fail) break;
        g_stage(sa, A, sam, sak, m0, M, kbeg + kc * kGk, kend, va_mode);
        g_stage(sb, B, sbn, sbk, n0, N, kbeg + kc * kGk, kend, vb_mode);
        // the staged tiles, written through the generic proxy, become visible
        // to the tensor cores' reads
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kk = 0; kk < kGk / 16; ++kk) {
                const uint32_t ko = kk * 2 * kTcLBO;    // one MMA's K = two core matrices
                g_mma(tmem, tc_desc(tc_smem(sa) + ko, kGsbo), tc_desc(tc_smem(sb) + ko, kGsbo),
                      (kc | kk) != 0);
            }
            tc_commit(&buf_bar[b]);
        }
    }
    // every MMA issued by this CTA has completed (also after a failed wait)
    if (tid == 0) tc_commit(&done_bar);
    if (!tc_mbar_wait(&done_bar, 0)) s_fail = 1;
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool fail = s_fail != 0;
    // accumulator lane = row: each 32-column block goes through shared memory
    // (the operand tiles are free now, rows padded to 33 words) so that the
    // warp writes each row's 32 columns with one coalesced store
    float *tp = (float *)(sm + (size_t)warp * 32 * 33 * 4);
    for (int q = 0; q < kGn / 32; ++q) {
        uint32_t v[32];
        const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(q * 32);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
            "%10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, "
            "%26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
              "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
              "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
              "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
              "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
              "=r"(v[30]), "=r"(v[31])
            : "r"(ta)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 32; ++j) tp[lane * 33 + j] = __uint_as_float(v[j]);
        __syncwarp();
        const int gn = n0 + q * 32 + lane;
        const float bv = (bias && gn < N) ? bias[gn] : 0.f;
        for (int r = 0; r < 32; ++r) {
            const int gm = m0 + warp * 32 + r;
            if (gm >= M || gn >= N) continue;
            float x = fail ? __int_as_float(0x7fc00000) : (nkc ? tp[r * 33 + lane] : 0.f);
            x += bv;
            C[gm * ldc + gn] = x;
            if (Cb)
                Cb[gm * ldc + gn] =
                    __bfloat16_as_ushort(__float2bfloat16_rn(relu ? fmaxf(x, 0.f) : x));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kGn)
                     : "memory");
}

// the split-K partials summed in slice order (fixed, so the result is the same
// on every run), then the bias and the BF16 copy as the GEMM's own epilogue
__global__ void k_gemm_splitk_sum(const float *__restrict__ part, int S, int M, int N,
                                  float *__restrict__ C, long ldc, uint16_t *__restrict__ Cb,
                                  const float *__restrict__ bias, int relu) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)M * N) return;
    const int m = (int)(i / N), n = (int)(i - (long)m * N);
    float x = 0.f;
    for (int z = 0; z < S; ++z) x += part[(long)z * M * N + i];
    if (bias) x += bias[n];
    C[m * ldc + n] = x;
    if (Cb) Cb[m * ldc + n] = __bfloat16_as_ushort(__float2bfloat16_rn(relu ? fmaxf(x, 0.f) : x));
}

// Slices of K for a product of few output tiles and a long K (the weight
// gradients, K = batch): at least 256 of K per slice, at most kGsplit slices,
// enough to give the GPU about 64 CTAs; partials need kGsplit M N floats.
constexpr int kGsplit = 16;

static int gemm_slices(int M, int N, int K) {
    const int tiles = ((M + kGm - 1) / kGm) * ((N + kGn - 1) / kGn);
    int S = 1;
    while (S < kGsplit && tiles * S < 64 && K / (2 * S) >= 256) S *= 2;
    return S;
}

static void gemm(const uint16_t *A, long sam, long sak, const uint16_t *B, long sbk, long sbn,
                 float *C, long ldc, uint16_t *Cb, const float *bias, int M, int N, int K,
                 int relu, cudaStream_t st, float *part = nullptr) {
    cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGsmem);
    const int S = part ? gemm_slices(M, N, K) : 1;
    if (S == 1) {
        dim3 grid((N + kGn - 1) / kGn, (M + kGm - 1) / kGm, 1);
        k_gemm_tc<<<grid, 128, kGsmem, st>>>(A, sam, sak, B, sbk, sbn, C, ldc, Cb, bias, M, N, K,
                                             relu, K);
        return;
    }
    // K slices a multiple of the 32-wide chunk
    const int kslice = ((K + S - 1) / S + kGk - 1) / kGk * kGk;
    dim3 grid((N + kGn - 1) / kGn, (M + kGm - 1) / kGm, S);
    k_gemm_tc<<<grid, 128, kGsmem, st>>>(A, sam, sak, B, sbk, sbn, part, N, nullptr, nullptr, M,
                                         N, K, 0, kslice);
    k_gemm_splitk_sum<<<(unsigned)(((long)M * N + 255) / 256), 256, 0, st>>>(part, S, M, N, C,
                                                                           ldc, Cb, bias, relu);
}

// ---------------------------------------------------------------- forward
// Z1[b][o] = b1[o] + f_b W1[nin][o] + sum over the sample's rows of W1[row][o]
__global__ void k_l1_fwd(chx_mlp_t P, const uint8_t *__restrict__ codes,
                         const float *__restrict__ lnbeta, const int *__restrict__ chain, int B,
                         float *__restrict__ Z1, uint16_t *__restrict__ H1b) {
    const int b = blockIdx.x, H = P.H, D2 = 2 * P.D, ns1 = P.nsp + 1;
    const int npt = P.nsp * (P.nsp - 1) / 2;
    if (b >= B) return;
    const uint8_t *cd = codes + (long)b * (D2 + 1);
    const float f = (lnbeta[b] - P.feat_shift) * P.feat_scale;
    const int ch = chain ? chain[b] : -1;
    const bool has_ch = ch >= 0 && ch < P.nchain;
    for (int o = threadIdx.x; o < H; o += blockDim.x) {
        float s = 0.f;
        for (int k = 0; k <= D2; ++k) {
            int row = k == 0 ? (int)cd[0] : npt + (k - 1) * ns1 + (int)cd[k];
            s += bf16f(P.W1[(long)row * H + o]);
        }
        if (has_ch) s += bf16f(P.W1[(long)(npt + D2 * ns1 + ch) * H + o]);
        s = fmaf(f, bf16f(P.W1[(long)P.nin * H + o]), P.b1[o]) + s;
        Z1[(long)b * H + o] = s;
        H1b[(long)b * H + o] = __bfloat16_as_ushort(__float2bfloat16_rn(fmaxf(s, 0.f)));
    }
}

// y[b] = b4 + sum_i h3[b][i] w4[i], one warp per sample
__global__ void k_out_fwd(chx_mlp_t P, const uint16_t *__restrict__ H3b, int B,
                          float *__restrict__ y) {
    const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (b >= B) return;
    float s = 0.f;
    for (int i = lane; i < P.H; i += 32)
        s = fmaf(bf16f(H3b[(long)b * P.H + i]), bf16f(P.w4[i]), s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[b] = s + P.b4[0];
}

// ---------------------------------------------------------------- backward
// dy_b = 2 (y_b - t_b) / B; dZ3 = BF16(dy_b w4[i] [Z3 > 0])
__global__ void k_out_back(chx_mlp_t P, const float *__restrict__ y, const float *__restrict__ t,
                           int B, const float *__restrict__ Z3, float *__restrict__ dy,
                           uint16_t *__restrict__ dZ3) {
    const int b = blockIdx.x;
    if (b >= B) return;
    const float d = 2.f * (y[b] - t[b]) / (float)B;
    if (threadIdx.x == 0) dy[b] = d;
    for (int i = threadIdx.x; i < P.H; i += blockDim.x) {
        long q = (long)b * P.H + i;
        float v = Z3[q] > 0.f ? d * bf16f(P.w4[i]) : 0.f;
        dZ3[q] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
}

// dZ = BF16(dH [Z > 0]), elementwise over n values
__global__ void k_relu_back(const float *__restrict__ dH, const float *__restrict__ Z, long n,
                            uint16_t *__restrict__ dZ) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    dZ[q] = __bfloat16_as_ushort(__float2bfloat16_rn(Z[q] > 0.f ? dH[q] : 0.f));
}

// out[o] = sum_b w_b X[b][o] (w NULL: 1), X BF16 (B, H): 32 columns per CTA,
// 8 row groups, reduced in fixed order
__global__ void __launch_bounds__(256) k_colsum(const uint16_t *__restrict__ X,
                                                const float *__restrict__ w, int B, int H,
                                                float *__restrict__ out) {
    __shared__ float red[8][33];
    const int cx = threadIdx.x & 31, ry = threadIdx.x >> 5;
    const int o = blockIdx.x * 32 + cx;
    float s = 0.f;
    if (o < H)
        for (int b = ry; b < B; b += 8) {
            float x = bf16f(X[(long)b * H + o]);
            s = w ? fmaf(w[b], x, s) : s + x;
        }
    red[ry][cx] = s;
    __syncthreads();
    if (ry == 0 && o < H) {
        float t = 0.f;
        for (int r = 0; r < 8; ++r) t += red[r][cx];
        out[o] = t;
    }
}

// gb4 = sum_b dy_b, loss = mean (y - t)^2 (one CTA, fixed order)
__global__ void __launch_bounds__(256) k_loss(const float *__restrict__ y,
                                              const float *__restrict__ t,
                                              const float *__restrict__ dy, int B,
                                              float *__restrict__ gb4, float *__restrict__ loss) {
    __shared__ float r1[256], r2[256];
    float s1 = 0.f, s2 = 0.f;
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        float e = y[b] - t[b];
        s1 = fmaf(e, e, s1);
        s2 += dy[b];
    }
    r1[threadIdx.x] = s1;
    r2[threadIdx.x] = s2;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            r1[threadIdx.x] += r1[threadIdx.x + h];
            r2[threadIdx.x] += r2[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *loss = r1[0] / (float)B;
        *gb4 = r2[0];
    }
}

// gW1: CTA k < 1 + 2D owns input site k: for each sample b the row named by
// code[b][k] gains dZ1[b][:]. A site's code values are below 8.
__global__ void __launch_bounds__(256) k_l1_back(chx_mlp_t P, const uint8_t *__restrict__ codes,
                                                 int B, const uint16_t *__restrict__ dZ1,
                                                 float *__restrict__ gW1) {
    const int k = blockIdx.x, H = P.H, D2 = 2 * P.D, ns1 = P.nsp + 1;
    const int npt = P.nsp * (P.nsp - 1) / 2;
    const int nv = k == 0 ? npt : ns1, row0 = k == 0 ? 0 : npt + (k - 1) * ns1;
    for (int o = threadIdx.x; o < H; o += blockDim.x) {
        float acc[8];
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[v] = 0.f;
        for (int b = 0; b < B; ++b) {
            const int v = codes[(long)b * (D2 + 1) + k];
            const float d = bf16f(dZ1[(long)b * H + o]);
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (u == v) acc[u] += d;
        }
        for (int v = 0; v < nv && v < 8; ++v) gW1[(long)(row0 + v) * H + o] = acc[v];
    }
}

// gW1 chain rows: CTA c sums dZ1 over the run of samples with chain c
// (chain sorted ascending), in order
__global__ void __launch_bounds__(256) k_chain_back(chx_mlp_t P, const int *__restrict__ chain,
                                                    int B, const uint16_t *__restrict__ dZ1,
                                                    float *__restrict__ gW1) {
    const int c = blockIdx.x, H = P.H;
    const int row = P.nsp * (P.nsp - 1) / 2 + 2 * P.D * (P.nsp + 1) + c;
    int lo = 0, hi = B;            // first sample with chain >= c
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (chain[mid] < c) lo = mid + 1;
        else hi = mid;
    }
    for (int o = threadIdx.x; o < H; o += blockDim.x) {
        float s = 0.f;
        for (int b = lo; b < B && chain[b] == c; ++b) s += bf16f(dZ1[(long)b * H + o]);
        gW1[(long)row * H + o] = s;
    }
}

__global__ void k_normfeat(chx_mlp_t P, const float *__restrict__ lnbeta, int B,
                           float *__restrict__ f) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < B) f[b] = (lnbeta[b] - P.feat_shift) * P.feat_scale;
}

// ---------------------------------------------------------------- predict
__global__ void __launch_bounds__(256) k_predict(const chx_mlp_t *__restrict__ Pd,
                                                 const uint8_t *__restrict__ codes,
                                                 const float *__restrict__ lnbeta,
                                                 const int *__restrict__ chain, int B,
                                                 float *__restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ chx_mlp_t P;
    if (threadIdx.x == 0) P = *Pd;
    __syncthreads();
    const int nsite = 2 * P.D + 1, nw = blockDim.x >> 5;
    float *part = (float *)smem;
    float *h = part + nw * P.H;
    uint8_t *s_codes = (uint8_t *)(h + P.H);
    for (int b = blockIdx.x; b < B; b += gridDim.x) {
        for (int k = threadIdx.x; k < nsite; k += blockDim.x)
            s_codes[k] = codes[(long)b * nsite + k];
        __syncthreads();
        float y = mlp_eval_cta(P, s_codes, lnbeta[b], chain ? chain[b] : -1, part, h);
        if (threadIdx.x == 0) out[b] = y;
        __syncthreads();
    }
}

// ---------------------------------------------------------------- Adam
__global__ void k_adam(float *__restrict__ w, uint16_t *__restrict__ wb,
                       const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       long n, float lr, float b1, float b2, float eps, float c1, float c2) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __bfloat16_as_ushort(__float2bfloat16_rn(wi));
}

struct MlpOffsets {
    int64_t W1, b1, W2, b2, W3, b3, w4, b4, n;
};
static MlpOffsets mlp_offsets(int nsp, int D, int nchain, int H) {
    MlpOffsets o;
    int64_t nin = mlp_nin(nsp, D, nchain);
    o.W1 = 0;
    o.b1 = o.W1 + (nin + 1) * H;
    o.W2 = o.b1 + H;
    o.b2 = o.W2 + (int64_t)H * H;
    o.W3 = o.b2 + H;
    o.b3 = o.W3 + (int64_t)H * H;
    o.w4 = o.b3 + H;
    o.b4 = o.w4 + H;
    o.n = o.b4 + 1;
    return o;
}

static bool mlp_shape_ok(int nsp, int D, int nchain, int H) {
    return nsp >= 2 && nsp <= 7 && D >= 1 && D <= 127 && nchain >= 0 && nchain <= (1 << 20) &&
           H >= 8 && H <= 256 && H % 8 == 0;
}

// dynamic shared memory of k_predict for the largest shape (H 256, D 127)
static size_t predict_smem_bytes() { return (size_t)(8 * 256 + 256) * sizeof(float) + 256; }

}  // namespace chx

using namespace chx;

extern "C" {

int64_t chx_mlp_nparam(int nsp, int D, int nchain, int H) {
    if (!mlp_shape_ok(nsp, D, nchain, H)) return -1;
    return mlp_offsets(nsp, D, nchain, H).n;
}

int chx_mlp_bind(chx_mlp_t *P, int nsp, int D, int nchain, int H, const float *theta,
                 const uint16_t *theta16) {
    CHX_REQUIRE(P && theta && theta16, "mlp_bind: null pointer");
    CHX_REQUIRE(mlp_shape_ok(nsp, D, nchain, H),
                "mlp_bind: need 2 <= nsp <= 7, 1 <= D <= 127, 0 <= nchain <= 2^20, "
                "8 <= H <= 256, H % 8 == 0");
    CHX_REQUIRE(nsp * (nsp - 1) / 2 <= 8, "mlp_bind: at most 8 species pairs");
    // W1, W2, W3 rows are read as 16-byte words
    CHX_REQUIRE(((uintptr_t)theta16 & 15) == 0, "mlp_bind: theta16 must be 16-byte aligned");
    MlpOffsets o = mlp_offsets(nsp, D, nchain, H);
    CHX_REQUIRE((o.W2 * 2) % 16 == 0 && (o.W3 * 2) % 16 == 0,
                "mlp_bind: layout misaligned for this H");
    P->nsp = nsp;
    P->D = D;
    P->H = H;
    P->nchain = nchain;
    P->nin = (int)mlp_nin(nsp, D, nchain);
    P->W1 = theta16 + o.W1;
    P->W2 = theta16 + o.W2;
    P->W3 = theta16 + o.W3;
    P->w4 = theta16 + o.w4;
    P->b1 = theta + o.b1;
    P->b2 = theta + o.b2;
    P->b3 = theta + o.b3;
    P->b4 = theta + o.b4;
    return CHX_OK;
}

int chx_mlp_predict(const chx_mlp_t *P, const uint8_t *codes, const float *lnbeta,
                    const int *chain, int B, float *out, void *stream) {
    CHX_REQUIRE(P && codes && lnbeta && out && B > 0, "mlp_predict: bad arguments");
    int grid = B < 148 * 8 ? B : 148 * 8;
    k_predict<<<grid, 256, predict_smem_bytes(), as_stream(stream)>>>(P, codes, lnbeta, chain, B,
                                                                      out);
    CHX_CHECK_LAUNCH("mlp_predict");
    return CHX_OK;
}

int64_t chx_mlp_work_bytes(int B, int H) {
    if (B <= 0 || H <= 0) return -1;
    const int64_t bh = (int64_t)B * H;
    return bh * (4 * 4 + 5 * 2) + (int64_t)B * 8 + (int64_t)kGsplit * H * H * 4 + 13 * 256;
}

int chx_mlp_grad(const chx_mlp_t *P, const uint8_t *codes, const float *lnbeta,
                 const int *chain, const float *target, int B, float *y, float *grad,
                 float *loss, void *work, void *stream) {
    CHX_REQUIRE(P && codes && lnbeta && target && y && grad && loss && work && B > 0,
                "mlp_grad: bad arguments");
    CHX_REQUIRE(mlp_shape_ok(P->nsp, P->D, P->nchain, P->H), "mlp_grad: bad shape");
    cudaStream_t st = as_stream(stream);
    const int H = P->H;
    const long bh = (long)B * H;
    const MlpOffsets of = mlp_offsets(P->nsp, P->D, P->nchain, H);
    auto take = [](char *&p, size_t n) {   // 256-byte aligned pieces of work
        char *r = p;
        p += (n + 255) / 256 * 256;
        return r;
    };
    char *p = (char *)work;
    float *Z1 = (float *)take(p, bh * 4), *Z2 = (float *)take(p, bh * 4),
          *Z3 = (float *)take(p, bh * 4), *dH = (float *)take(p, bh * 4);
    uint16_t *H1b = (uint16_t *)take(p, bh * 2), *H2b = (uint16_t *)take(p, bh * 2),
             *H3b = (uint16_t *)take(p, bh * 2);
    uint16_t *dZa = (uint16_t *)take(p, bh * 2), *dZb = (uint16_t *)take(p, bh * 2);
    float *dy = (float *)take(p, (size_t)B * 4), *f = (float *)take(p, (size_t)B * 4);
    float *part = (float *)take(p, (size_t)kGsplit * H * H * 4);   // split-K partials
    if ((int64_t)(p - (char *)work) > chx_mlp_work_bytes(B, H)) {
        set_error("mlp_grad: work carve-up exceeds chx_mlp_work_bytes");
        return CHX_ERR_SCRATCH;
    }
    const chx_mlp_t Pv = *P;
    // forward
    k_l1_fwd<<<B, 256, 0, st>>>(Pv, codes, lnbeta, chain, B, Z1, H1b);
    gemm(H1b, H, 1, P->W2, H, 1, Z2, H, H2b, P->b2, B, H, H, 1, st);
    gemm(H2b, H, 1, P->W3, H, 1, Z3, H, H3b, P->b3, B, H, H, 1, st);
    k_out_fwd<<<(B + 7) / 8, 256, 0, st>>>(Pv, H3b, B, y);
    // output layer
    k_out_back<<<B, 256, 0, st>>>(Pv, y, target, B, Z3, dy, dZa);
    k_loss<<<1, 256, 0, st>>>(y, target, dy, B, grad + of.b4, loss);
    const int cs = (H + 31) / 32;
    k_colsum<<<cs, 256, 0, st>>>(H3b, dy, B, H, grad + of.w4);
    // layer 3: gW3 = H2^T dZ3, gb3, dH2 = dZ3 W3^T
    gemm(H2b, 1, H, dZa, H, 1, grad + of.W3, H, nullptr, nullptr, H, H, B, 0, st, part);
    k_colsum<<<cs, 256, 0, st>>>(dZa, nullptr, B, H, grad + of.b3);
    gemm(dZa, H, 1, P->W3, 1, H, dH, H, nullptr, nullptr, B, H, H, 0, st);
    k_relu_back<<<(unsigned)((bh + 255) / 256), 256, 0, st>>>(dH, Z2, bh, dZb);
    // layer 2
    gemm(H1b, 1, H, dZb, H, 1, grad + of.W2, H, nullptr, nullptr, H, H, B, 0, st, part);
    k_colsum<<<cs, 256, 0, st>>>(dZb, nullptr, B, H, grad + of.b2);
    gemm(dZb, H, 1, P->W2, 1, H, dH, H, nullptr, nullptr, B, H, H, 0, st);
    k_relu_back<<<(unsigned)((bh + 255) / 256), 256, 0, st>>>(dH, Z1, bh, dZa);
    // layer 1
    k_colsum<<<cs, 256, 0, st>>>(dZa, nullptr, B, H, grad + of.b1);
    k_normfeat<<<(B + 255) / 256, 256, 0, st>>>(Pv, lnbeta, B, f);
    k_colsum<<<cs, 256, 0, st>>>(dZa, f, B, H, grad + of.W1 + (int64_t)P->nin * H);
    k_l1_back<<<2 * P->D + 1, 256, 0, st>>>(Pv, codes, B, dZa, grad + of.W1);
    if (P->nchain > 0) {
        if (chain) {
            k_chain_back<<<P->nchain, 256, 0, st>>>(Pv, chain, B, dZa, grad + of.W1);
        } else {
            const int64_t r0 = (int64_t)(P->nin - P->nchain) * H;
            cudaError_t e = cudaMemsetAsync(grad + of.W1 + r0, 0,
                                            sizeof(float) * (size_t)P->nchain * H, st);
            if (e != cudaSuccess) return cuda_fail(e, "mlp_grad memset");
        }
    }
    CHX_CHECK_LAUNCH("mlp_grad");
    return CHX_OK;
}

int chx_mlp_adam(float *theta, uint16_t *theta16, const float *grad, float *m, float *v,
                 int64_t n, float lr, float beta1, float beta2, float eps, int t, void *stream) {
    CHX_REQUIRE(theta && theta16 && grad && m && v && n > 0 && t >= 1, "mlp_adam: bad arguments");
    const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
    k_adam<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(
        theta, theta16, grad, m, v, (long)n, lr, beta1, beta2, eps, c1, c2);
    CHX_CHECK_LAUNCH("mlp_adam");
    return CHX_OK;
}

}  // extern "C"
