// chx_ft_tc.cu -- the windowed FT contraction out = chi . B on the tcgen05
// tensor cores (A5, precisions 2 and 3 of chx_ft_batch).
//
// Split-BF16 (precision 2): each FP64 operand x is split into two BF16
// numbers, x_hi = bf16(x) and x_lo = bf16(x - x_hi); a product a.b is taken
// as a_hi b_hi + a_hi b_lo + a_lo b_hi (the a_lo b_lo term is below 2^-16 of
// it), three BF16 MMAs (kind::f16) with FP32 accumulation in tensor memory,
// which keeps about 16 significant bits per product where one BF16 product
// keeps 8. TF32 (precision 3): the operands rounded to TF32 (10-bit
// mantissa), one MMA (kind::tf32) per product, FP32 accumulation.
//
// Layout. Both operands are split by a pre-pass (k_tc_split: the basis,
// 2 nR x nk transposed, and chi, rows x nk) into 128 x 32 tiles in scratch
// (hi and lo BF16, or TF32), each already in the no-swizzle K-major
// shared-memory layout the MMA reads: 8 x 16-byte core matrices, 128 B apart
// along K and one row group (K bytes / 16 core matrices) apart along rows;
// one thread of the pre-pass writes one 16-byte core-matrix row.
// The main kernel (k_ft_tc, one 128 x 128 output tile per CTA, three CTAs per
// SM) runs a two-stage ring over 32-wide K chunks driven by one thread: the
// chunk's A and B tiles arrive by bulk-async copies (cp.async.bulk, no
// multicast) completing on the stage's mbarrier, the chunk's MMAs (6 of
// 128 x 128 x 16 BF16, or 4 of 128 x 128 x 8 TF32) go into one 128 x 128 FP32
// accumulator in tensor memory and commit to the stage's second mbarrier,
// and the stage is refilled with the chunk two ahead once they are done.
// Four warps finally read the accumulator (lane = row) with tcgen05.ld, turn
// each 32 x 32 block around in shared memory and write FP64 rows with
// coalesced stores.
//
// Every wait is bounded (kTcSpin polls); a wait that runs out sets the error
// word in the first 4 bytes of scratch (CHX_DEVERR_INDEX), waits (bounded)
// for the copies and MMAs it started, frees its tensor memory and returns.
#include <cuda_bf16.h>
#include "chx_common.cuh"

namespace chx {

constexpr int kTcM = 128, kTcN = 128, kTcK = 32;        // CTA tile and K chunk
constexpr int kTcStages = 2;                           // copy/MMA ring depth
constexpr uint32_t kTcLBO = 128;                        // core matrices along K (bytes)
constexpr int kTcSpin = 1 << 24;
constexpr int kTcTmemCols = kTcN;                       // FP32 accumulator columns

// Operand modes: split-BF16 (two BF16 parts of 2 bytes, MMA K = 16, kind::f16
// with A and B BF16) and TF32 (one 4-byte part, MMA K = 8, kind::tf32); both
// D FP32, A and B K-major, N = M = 128 in the instruction descriptor.
template <bool TF32>
struct TcMode {
    static constexpr int esz = TF32 ? 4 : 2, parts = TF32 ? 1 : 2, kmma = TF32 ? 8 : 16;
    static constexpr uint32_t sbo = (uint32_t)(kTcK * esz / 16) * 128;   // row group stride
    static constexpr uint32_t tileA = kTcM * kTcK * esz, tileB = kTcN * kTcK * esz;
    static constexpr uint32_t stage = parts * (tileA + tileB);
    static constexpr uint32_t fmt = TF32 ? 2u : 1u;
    static constexpr uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) |
                                      ((uint32_t)(kTcN >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
    static constexpr size_t smem = (size_t)kTcStages * stage + 1024;
    // byte offset of element (r, k) inside one operand tile of kTcK values
    static __host__ __device__ __forceinline__ uint32_t off(int r, int k) {
        return (uint32_t)((r >> 3) * sbo + (k * esz / 16) * kTcLBO + (r & 7) * 16 +
                          (k * esz) % 16);
    }
};

__device__ __forceinline__ uint32_t tc_smem(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: start address, leading (K) and stride
// (row-group) byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)(kTcLBO >> 4) << 16) |
           ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(bar)) : "memory");
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

__device__ __forceinline__ void tc_load_tile(void *dst, const void *src, uint32_t bytes,
                                             uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(tc_smem(dst)),
        "l"(src), "r"(bytes), "r"(tc_smem(bar))
        : "memory");
}

__device__ __forceinline__ void tc_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc_smem(bar)),
                 "r"(bytes)
                 : "memory");
}

template <bool TF32>
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc) {
    if constexpr (TF32)
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::
                "r"(tmem),
            "l"(da), "l"(db), "r"(TcMode<true>::idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u),
            "r"(0u)
            : "memory");
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::
                "r"(tmem),
            "l"(da), "l"(db), "r"(TcMode<false>::idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u),
            "r"(0u)
            : "memory");
}

// x rounded to TF32 (nearest, ties away), kept in an FP32 container
__device__ __forceinline__ uint32_t tc_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            tc_smem(bar))
        : "memory");
}

// One operand of the contraction: X (R x C, element (r, c) at X[r*sr + c*sc])
// zero-padded to Rp x Kp, and where its parts go.
struct TcSplitJob {
    const double *X;
    int R, C, Rp;
    long sr, sc;
    uint8_t *hi, *lo;
};

// The operand parts of both jobs (the basis in blocks [0, nblk_a), chi in the
// rest), written as 128 x 32 tiles (tile (rt, kt) at (rt * Kp/32 + kt)): hi
// and lo BF16, or TF32 into hi. One thread takes 8 consecutive k of one row (a
// 16-byte row of a core matrix in BF16, two in TF32) and threads run
// row-fastest, so that rows of chi (k contiguous) and columns of the basis
// (rows contiguous) are both read coalesced and every store is 16 bytes.
// Block 0 also clears the error word of the contraction that follows, which
// is launched as a programmatic dependent of this grid.
template <bool TF32>
__global__ void k_tc_split(TcSplitJob ja, TcSplitJob jb, int Kp, int nblk_a, int *err) {
    typedef TcMode<TF32> Md;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (blockIdx.x == 0 && threadIdx.x == 0) *err = 0;
    const bool first = (int)blockIdx.x < nblk_a;
    const TcSplitJob &J = first ? ja : jb;
    const long blk = first ? blockIdx.x : blockIdx.x - nblk_a;
    const long nblk = first ? nblk_a : gridDim.x - nblk_a;
    const double *__restrict__ X = J.X;
    const int R = J.R, C = J.C, Rp = J.Rp;
    const long sr = J.sr, sc = J.sc;
    uint8_t *__restrict__ hi = J.hi;
    uint8_t *__restrict__ lo = J.lo;
    const int ng = Kp / 8;
    const long n = (long)Rp * ng;
    for (long q = blk * blockDim.x + threadIdx.x; q < n; q += nblk * blockDim.x) {
        const int r = (int)(q % Rp), k0 = (int)(q / Rp) * 8;
        double x[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            x[j] = (r < R && k0 + j < C) ? X[r * sr + (long)(k0 + j) * sc] : 0.0;
        const long tile = ((long)(r / kTcN) * (Kp / kTcK) + k0 / kTcK) * Md::tileB;
        const int rr = r % kTcN, kk = k0 % kTcK;
        if constexpr (TF32) {
            uint4 a, b;
            a.x = tc_tf32((float)x[0]); a.y = tc_tf32((float)x[1]);
            a.z = tc_tf32((float)x[2]); a.w = tc_tf32((float)x[3]);
            b.x = tc_tf32((float)x[4]); b.y = tc_tf32((float)x[5]);
            b.z = tc_tf32((float)x[6]); b.w = tc_tf32((float)x[7]);
            *(uint4 *)(hi + tile + Md::off(rr, kk)) = a;
            *(uint4 *)(hi + tile + Md::off(rr, kk + 4)) = b;
        } else {
            __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                h[j] = __double2bfloat16(x[j]);
                l[j] = __double2bfloat16(x[j] - (double)__bfloat162float(h[j]));
            }
            *(uint4 *)(hi + tile + Md::off(rr, kk)) = *(const uint4 *)h;
            *(uint4 *)(lo + tile + Md::off(rr, kk)) = *(const uint4 *)l;
        }
    }
}

template <bool TF32>
__global__ void __launch_bounds__(128, 3) k_ft_tc(const uint8_t *__restrict__ Ahi,
                                                  const uint8_t *__restrict__ Alo, int rows,
                                                  const uint8_t *__restrict__ Bhi,
                                                  const uint8_t *__restrict__ Blo, int nkt,
                                                  int ncol, double *__restrict__ out,
                                                  int *__restrict__ err) {
    extern __shared__ uint8_t tc_raw[];
    __shared__ __align__(8) uint64_t full[kTcStages], freed[kTcStages], done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    uint8_t *ring = (uint8_t *)(((uintptr_t)tc_raw + 1023) & ~(uintptr_t)1023);
    typedef TcMode<TF32> Md;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nt = blockIdx.x, mt = blockIdx.y;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         tc_smem(&s_tmem)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < kTcStages; ++s) {
            tc_mbar_init(&full[s]);
            tc_mbar_init(&freed[s]);
        }
        tc_mbar_init(&done);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    // the operand parts and the cleared error word come from the split grid
    // this launch may overlap: everything below waits for it to complete
    asm volatile("griddepcontrol.wait;" ::: "memory");

    const long tstride = (long)nkt * Md::tileB;              // one row of tiles
    const uint8_t *b_hi = Bhi + nt * tstride, *b_lo = Blo + nt * tstride;
    const uint8_t *a_hi = Ahi + mt * tstride, *a_lo = Alo + mt * tstride;
    const int row0 = mt * kTcM;
    // Thread 0 runs the pipeline: the operand parts of chunk kt (A and B, hi
    // and lo, split in advance into the tiles' shared-memory image) arrive by
    // bulk copies into stage kt % S, the MMAs of chunk kt are issued when they
    // have landed, and the stage is refilled with chunk kt + S as soon as
    // those MMAs are done, so the copies of the next S - 1 chunks overlap the
    // MMAs of this one. Every wait is bounded; a failed wait ends the loop and
    // the copies still owed are waited for before the CTA moves on.
    if (tid == 0) {
        int issued[kTcStages] = {}, landed[kTcStages] = {};
        auto issue = [&](int kt) {
            const int s = kt % kTcStages;
            uint8_t *st = ring + (size_t)s * Md::stage;
            uint8_t *sb = st + Md::parts * Md::tileA;
            tc_expect(&full[s], Md::parts * (Md::tileA + Md::tileB));
            tc_load_tile(st, a_hi + (long)kt * Md::tileA, Md::tileA, &full[s]);
            tc_load_tile(sb, b_hi + (long)kt * Md::tileB, Md::tileB, &full[s]);
            if (!TF32) {
                tc_load_tile(st + Md::tileA, a_lo + (long)kt * Md::tileA, Md::tileA, &full[s]);
                tc_load_tile(sb + Md::tileB, b_lo + (long)kt * Md::tileB, Md::tileB, &full[s]);
            }
            ++issued[s];
        };
        for (int kt = 0; kt < nkt && kt < kTcStages; ++kt) issue(kt);
        int ok = 1;
        for (int kt = 0; kt < nkt && ok; ++kt) {
            const int s = kt % kTcStages;
            const uint32_t par = (uint32_t)((kt / kTcStages) & 1);
            if (!tc_mbar_wait(&full[s], par)) {
                ok = 0;
                break;
            }
            ++landed[s];
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t base = tc_smem(ring + (size_t)s * Md::stage);
            const uint32_t bbase = base + Md::parts * Md::tileA;
#pragma unroll
            for (int kk = 0; kk < kTcK / Md::kmma; ++kk) {
                const uint32_t ko = kk * 2 * kTcLBO;       // one MMA's K = two core matrices
                const uint64_t ahi = tc_desc(base + ko, Md::sbo);
                const uint64_t bhi = tc_desc(bbase + ko, Md::sbo);
                tc_mma<TF32>(tmem, ahi, bhi, (kt | kk) != 0);
                if constexpr (!TF32) {
                    const uint64_t alo = tc_desc(base + Md::tileA + ko, Md::sbo);
                    const uint64_t blo = tc_desc(bbase + Md::tileB + ko, Md::sbo);
                    tc_mma<TF32>(tmem, ahi, blo, 1u);
                    tc_mma<TF32>(tmem, alo, bhi, 1u);
                }
            }
            tc_commit(&freed[s]);
            if (kt + kTcStages < nkt) {
                if (!tc_mbar_wait(&freed[s], par)) {
                    ok = 0;
                    break;
                }
                issue(kt + kTcStages);
            }
        }
        if (!ok) s_fail = 1;
        tc_commit(&done);
        for (int s = 0; s < kTcStages; ++s)
            for (int w = landed[s]; w < issued[s]; ++w)
                if (!tc_mbar_wait(&full[s], (uint32_t)(w & 1))) break;
        if (!tc_mbar_wait(&done, 0)) s_fail = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (!s_fail) {
        // each warp turns its 32 x 32 block around in shared memory (the ring
        // is free now) so that every store writes 32 consecutive doubles
        float *tb = (float *)ring + warp * 32 * 33;
#pragma unroll 1
        for (int c0 = 0; c0 < kTcN; c0 += 32) {
            uint32_t v[32];
            const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
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
#pragma unroll
            for (int j = 0; j < 32; ++j) tb[lane * 33 + j] = __uint_as_float(v[j]);
            __syncwarp();
            const int col = nt * kTcN + c0 + lane;
#pragma unroll 4
            for (int r = 0; r < 32; ++r) {
                const int row = row0 + warp * 32 + r;
                if (row < rows && col < ncol) out[(long)row * ncol + col] = (double)tb[r * 33 + lane];
            }
            __syncwarp();
        }
    } else if (tid == 0) {
        atomicOr(err, CHX_DEVERR_INDEX);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTcTmemCols)
                     : "memory");
}

struct TcPlan {
    int Mp, Np, Kp;
    size_t a_bytes, b_bytes, total;
};
// scratch: an error word, then the operand parts of the basis and of chi,
// each split into the tiles' shared-memory image
static TcPlan tc_plan(int rows, int nk, int nR, bool tf32) {
    TcPlan p;
    p.Mp = (rows + kTcM - 1) / kTcM * kTcM;
    p.Np = (2 * nR + kTcN - 1) / kTcN * kTcN;
    p.Kp = (nk + kTcK - 1) / kTcK * kTcK;
    p.a_bytes = (size_t)p.Mp * p.Kp * (tf32 ? 4 : 2);
    p.b_bytes = (size_t)p.Np * p.Kp * (tf32 ? 4 : 2);
    p.total = 256 + (tf32 ? 1 : 2) * (p.a_bytes + p.b_bytes);
    return p;
}

int64_t ft_batch_tc_scratch(int rows, int nk, int nR, bool tf32) {
    return (int64_t)tc_plan(rows, nk, nR, tf32).total;
}

template <bool TF32>
static int ft_batch_tc_mode(const double *chi, int rows, int nk, const double *basis, int nR,
                            double *out, void *scratch, int64_t scratch_bytes, cudaStream_t st) {
    typedef TcMode<TF32> Md;
    const TcPlan p = tc_plan(rows, nk, nR, TF32);
    CHX_REQUIRE(scratch && scratch_bytes >= (int64_t)p.total,
                "ft_batch: the tensor-core path needs %zu bytes of scratch", p.total);
    CHX_REQUIRE(((uintptr_t)scratch & 255) == 0, "ft_batch: scratch must be 256-byte aligned");
    uint8_t *base = (uint8_t *)scratch;
    int *err = (int *)base;
    const int parts = TF32 ? 1 : 2;
    uint8_t *bhi = base + 256, *bl = bhi + p.b_bytes;
    uint8_t *ahi = base + 256 + parts * p.b_bytes, *al = ahi + p.a_bytes;
    const int ncol = 2 * nR;
    // both operands split by one launch: the basis (its columns are the rows
    // of B) in the first blocks, chi in the rest
    const TcSplitJob jb = {basis, ncol, nk, p.Np, 1, ncol, bhi, bl};
    const TcSplitJob ja = {chi, rows, nk, p.Mp, nk, 1, ahi, al};
    const long nb = (long)p.Np * p.Kp / 8, na = (long)p.Mp * p.Kp / 8;
    const int gb = (int)std::min<long>((nb + 255) / 256, 592);
    const int ga = (int)std::min<long>((na + 255) / 256, 1184);
    k_tc_split<TF32><<<gb + ga, 256, 0, st>>>(jb, ja, p.Kp, gb, err);
    CHX_CHECK_LAUNCH("ft_batch split");
    cudaError_t e = cudaFuncSetAttribute(k_ft_tc<TF32>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)Md::smem);
    if (e != cudaSuccess) return cuda_fail(e, "ft_batch tc attribute");
    // a programmatic dependent of the split: its prologue (barriers, tensor
    // memory) overlaps the split's tail, its loads wait for the split's end
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p.Np / kTcN, p.Mp / kTcM);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = Md::smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_ft_tc<TF32>, (const uint8_t *)ahi, (const uint8_t *)al, rows,
                           (const uint8_t *)bhi, (const uint8_t *)bl, p.Kp / kTcK, ncol, out,
                           err);
    if (e != cudaSuccess) return cuda_fail(e, "ft_batch tc launch");
    CHX_CHECK_LAUNCH("ft_batch tc");
    return CHX_OK;
}

int ft_batch_tc(const double *chi, int rows, int nk, const double *basis, int nR, double *out,
                void *scratch, int64_t scratch_bytes, cudaStream_t st, bool tf32) {
    return tf32 ? ft_batch_tc_mode<true>(chi, rows, nk, basis, nR, out, scratch, scratch_bytes, st)
                : ft_batch_tc_mode<false>(chi, rows, nk, basis, nR, out, scratch, scratch_bytes,
                                          st);
}

}  // namespace chx
