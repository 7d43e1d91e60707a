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
// Layout. Both operands are split by a pre-pass (k_tc_split, one launch for
// both: the basis, 2 nR x nk transposed, and chi, rows x nk) into 128 x 32
// tiles in scratch (hi and lo BF16, or TF32), each already in the no-swizzle
// K-major shared-memory layout the MMA reads: 8 x 16-byte core matrices,
// 128 B apart along K and one row group (K bytes / 16 core matrices) apart
// along rows.
// The contraction (k_ft_tc) is persistent, one CTA per SM over the 128 x 128
// output tiles, and launched as a programmatic dependent of the split. One
// thread streams 32-wide K chunks by bulk-async copies (cp.async.bulk, no
// multicast) through a ring of stages; one thread issues each chunk's MMAs
// (6 of 128 x 128 x 16 BF16, or 4 of 128 x 128 x 8 TF32) into one of two
// 128-column FP32 accumulators in tensor memory; four warps read the other
// accumulator (lane = row, tcgen05.ld), stage 32 x 16 FP64 boxes in shared
// memory and write chi(R) by TMA tensor stores, so that one tile's stores
// overlap the next tile's MMAs. With nk <= 256 every CTA keeps one column
// tile of the basis resident in shared memory and streams only chi.
//
// Every wait is bounded (kTcSpin polls); a wait that runs out sets the error
// word in the first 4 bytes of scratch (CHX_DEVERR_INDEX), waits (bounded)
// for the copies and MMAs it started, frees its tensor memory and returns.
#include <cuda.h>
#include <cstring>
#include <cuda_bf16.h>
#include "chx_common.cuh"
#include "chx_tc.cuh"

namespace chx {

constexpr int kTcM = 128, kTcN = 128, kTcK = 32;        // CTA tile and K chunk
constexpr int kTcStages = 5;                           // ring depth, both operands streamed
constexpr int kTcStagesRes = 4;                        // ring depth, chi only (basis resident)
constexpr int kTcResKp = 256;                          // largest padded nk kept resident
constexpr int kTcBox = 32 * 16 * 8;                     // one staged chi(R) box: 32 rows x 16 FP64
constexpr int kTcAcc = 2;                              // accumulators in tensor memory
constexpr int kTcThreads = 192;                        // 4 epilogue warps, producer, MMA
constexpr int kTcTmemCols = kTcAcc * kTcN;              // FP32 accumulator columns

// Operand modes: split-BF16 (two BF16 parts of 2 bytes, MMA K = 16, kind::f16
// with A and B BF16) and TF32 (one 4-byte part, MMA K = 8, kind::tf32); both
// D FP32, A and B K-major, N = M = 128 in the instruction descriptor.
template <bool TF32>
struct TcMode {
    static constexpr int esz = TF32 ? 4 : 2, parts = TF32 ? 1 : 2, kmma = TF32 ? 8 : 16;
    static constexpr uint32_t sbo = (uint32_t)(kTcK * esz / 16) * 128;   // row group stride
    static constexpr uint32_t tileA = kTcM * kTcK * esz, tileB = kTcN * kTcK * esz;
    static constexpr uint32_t stage = parts * (tileA + tileB);   // both operands of a chunk
    static constexpr uint32_t stage_a = parts * tileA;           // chi's parts of a chunk
    static constexpr uint32_t fmt = TF32 ? 2u : 1u;
    static constexpr uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) |
                                      ((uint32_t)(kTcN >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
    // shared memory: the stage ring, two staged chi(R) boxes per epilogue
    // warp, the resident basis tile (all nkt chunks) when RES, alignment
    static size_t smem(bool res, int nkt) {
        return res ? (size_t)kTcStagesRes * stage_a + 4 * 2 * kTcBox +
                         (size_t)parts * nkt * tileB + 1024
                   : (size_t)kTcStages * stage + 4 * 2 * kTcBox + 1024;
    }
    // both layouts at their largest fit the 227 KB a CTA may opt into (less
    // the static barriers)
    static_assert((size_t)kTcStagesRes * stage_a + 4 * 2 * kTcBox +
                          (size_t)parts * (kTcResKp / kTcK) * tileB + 1024 <= 232448 - 256,
                  "resident-basis layout exceeds shared memory");
    static_assert((size_t)kTcStages * stage + 4 * 2 * kTcBox + 1024 <= 232448 - 256,
                  "streaming layout exceeds shared memory");
    // byte offset of element (r, k) inside one operand tile of kTcK values
    static __host__ __device__ __forceinline__ uint32_t off(int r, int k) {
        return (uint32_t)((r >> 3) * sbo + (k * esz / 16) * kTcLBO + (r & 7) * 16 +
                          (k * esz) % 16);
    }
};

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
// 16-byte row of a core matrix in BF16, two in TF32); one warp takes 8 rows x
// 32 k (lane = row + 8 x k group), so that it reads 256-byte runs of the rows
// of chi (64-byte runs of the basis columns) and writes one row group of one
// tile, 512 contiguous bytes in BF16 (1 KB in TF32).
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
    const long n = (long)Rp * (Kp / 8);                      // Rp, Kp: multiples of 128, 32
    const int nrg = Rp / 8;
    for (long q = blk * blockDim.x + threadIdx.x; q < n; q += nblk * blockDim.x) {
        const long w = q >> 5;
        const int l = (int)(q & 31);
        const int r = (int)(w % nrg) * 8 + (l & 7), k0 = (int)(w / nrg) * 32 + (l >> 3) * 8;
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

// Bounded wait that also gives up as soon as another role of the CTA has
// recorded a failure in *fail.
__device__ __forceinline__ bool tc_mbar_wait_or_fail(uint64_t *bar, uint32_t parity,
                                                     const volatile int *fail) {
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
        if (*fail) return false;
    }
    return false;
}

// Persistent contraction: one CTA per SM walks the output tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... (tile t = row tile t / ntn, column tile t % ntn).
// Warp 4 lane 0 (producer) streams the operand chunks of all its tiles through
// the stage ring, warp 5 lane 0 (MMA) accumulates tile i into tensor-memory
// accumulator i % 2, and warps 0-3 drain accumulator (i - 1) % 2 into chi(R)
// meanwhile, so that the FP64 stores of one tile overlap the MMAs of the next.
// Barriers: full[s] (chunk landed, producer -> MMA), freed[s] (its MMAs done,
// MMA -> producer), acc_full[b] (tile accumulated, MMA -> epilogue) and
// acc_empty[b] (accumulator read out, the four epilogue warps -> MMA).
// RES: every CTA keeps one column tile (tc_tile) and its basis parts, loaded
// with the chunks of its first tile, stay resident in shared memory; only
// chi's parts stream through the ring after that, which halves the bytes a
// tile moves from L2 into the SM (the bound of the main loop).
template <bool RES>
__device__ __forceinline__ bool tc_tile(int i, int ntn, int mtiles, int &mt, int &nt) {
    const int G = gridDim.x, c = blockIdx.x;
    if (RES) {
        nt = c % ntn;
        mt = c / ntn + i * ((G - 1 - nt) / ntn + 1);         // this column's CTAs share its rows
        return mt < mtiles;
    }
    const int t = c + i * G;
    mt = t / ntn;
    nt = t % ntn;
    return t < ntn * mtiles;
}

// The window sums of the fused form (SUMS): instead of chi(R), each row's
// sums against the target t and weights w over the tile's bins (w is 0
// outside the fit window, so they run over it), anchored at a scale s0:
// Re<m,t>, <m,m>, R = sum w |s0 m - t|^2, Q = sum w Re(m (s0 m - t)*),
// P = sum w |m|^2, and the unweighted Ru = sum |s0 m - t|^2 and
// Qu = sum Re(m (s0 m - t)*), into part[(row * ntn + nt) * kSums]; then
// sum w |s m - t|^2 = R + 2 (s - s0) Q + (s - s0)^2 P for any scale s (and
// the R-factor's numerator Ru + 2 (s - s0) Qu + (s - s0)^2 <m,m>), the
// residual at s0 carrying its size without cancelling.
constexpr int kSums = 7;
struct TcSums {
    const double *tgt;   // (nR, 2) target chi(R), re/im
    const double *wgt;   // (nR) 1 / sigma^2 on the fit window, 0 elsewhere
    double *part;        // (rows, ntn, kSums)
    int nR;
    double s0;
};

template <bool TF32, bool RES, bool SUMS>
__global__ void __launch_bounds__(kTcThreads, 1) k_ft_tc(const uint8_t *__restrict__ Ahi,
                                                         const uint8_t *__restrict__ Alo,
                                                         int rows,
                                                         const uint8_t *__restrict__ Bhi,
                                                         const uint8_t *__restrict__ Blo,
                                                         int nkt, int ncol, int ntn, int mtiles,
                                                         const __grid_constant__ CUtensorMap tm_out,
                                                         TcSums sums, int *__restrict__ err) {
    extern __shared__ uint8_t tc_raw[];
    __shared__ __align__(8) uint64_t full[kTcStages], freed[kTcStages], acc_full[kTcAcc],
        acc_empty[kTcAcc], done;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_fail;
    uint8_t *ring = (uint8_t *)(((uintptr_t)tc_raw + 1023) & ~(uintptr_t)1023);
    typedef TcMode<TF32> Md;
    constexpr int S = RES ? kTcStagesRes : kTcStages;
    constexpr uint32_t SB = RES ? Md::stage_a : Md::stage;    // bytes of one ring stage
    uint8_t *bres = ring + (size_t)S * SB + 4 * 2 * kTcBox;   // resident basis (RES)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         tc_smem(&s_tmem)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 128) {
        for (int s = 0; s < S; ++s) {
            tc_mbar_init(&full[s], 1);
            tc_mbar_init(&freed[s], 1);
        }
        for (int b = 0; b < kTcAcc; ++b) {
            tc_mbar_init(&acc_full[b], 1);
            tc_mbar_init(&acc_empty[b], 4);
        }
        tc_mbar_init(&done, 1);
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

    const long tstride = (long)nkt * Md::tileB;              // one row of tiles (tileA == tileB)
    if (warp == 4) {
        if (lane == 0) {
            // producer: chunk c (over all tiles of this CTA) into stage c % S,
            // once the MMAs of the chunk S before it have released the stage
            int issued[kTcStages] = {};
            long c = 0;
            bool ok = true;
            int mt, nt;
            for (int i = 0; ok && tc_tile<RES>(i, ntn, mtiles, mt, nt); ++i) {
                const uint8_t *a_hi = Ahi + mt * tstride, *a_lo = Alo + mt * tstride;
                const uint8_t *b_hi = Bhi + nt * tstride, *b_lo = Blo + nt * tstride;
                const bool with_b = !RES || i == 0;           // the basis chunk comes along
                for (int kt = 0; kt < nkt; ++kt, ++c) {
                    const int s = (int)(c % S);
                    const long u = c / S;
                    if (u > 0 && !tc_mbar_wait_or_fail(&freed[s], (uint32_t)((u - 1) & 1), &s_fail)) {
                        ok = false;
                        break;
                    }
                    uint8_t *st = ring + (size_t)s * SB;
                    uint8_t *sb = RES ? bres + (size_t)kt * Md::parts * Md::tileB
                                      : st + Md::parts * Md::tileA;
                    tc_expect(&full[s], Md::parts * (Md::tileA + (with_b ? Md::tileB : 0u)));
                    tc_load_tile(st, a_hi + (long)kt * Md::tileA, Md::tileA, &full[s]);
                    if (!TF32)
                        tc_load_tile(st + Md::tileA, a_lo + (long)kt * Md::tileA, Md::tileA,
                                     &full[s]);
                    if (with_b) {
                        tc_load_tile(sb, b_hi + (long)kt * Md::tileB, Md::tileB, &full[s]);
                        if (!TF32)
                            tc_load_tile(sb + Md::tileB, b_lo + (long)kt * Md::tileB, Md::tileB,
                                         &full[s]);
                    }
                    ++issued[s];
                }
            }
            if (!ok) s_fail = 1;
            // at most the last fill of each stage can still be in flight
            for (int s = 0; s < S; ++s)
                if (issued[s] && !tc_mbar_wait(&full[s], (uint32_t)((issued[s] - 1) & 1)))
                    s_fail = 1;
        }
    } else if (warp == 5) {
        if (lane == 0) {
            long c = 0;
            bool ok = true;
            int mt, nt;
            for (int i = 0; ok && tc_tile<RES>(i, ntn, mtiles, mt, nt); ++i) {
                const int b = i & 1, ub = i >> 1;
                if (ub > 0 &&
                    !tc_mbar_wait_or_fail(&acc_empty[b], (uint32_t)((ub - 1) & 1), &s_fail)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(b * kTcN);
                for (int kt = 0; kt < nkt; ++kt, ++c) {
                    const int s = (int)(c % S);
                    const long u = c / S;
                    if (!tc_mbar_wait_or_fail(&full[s], (uint32_t)(u & 1), &s_fail)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t base = tc_smem(ring + (size_t)s * SB);
                    const uint32_t bbase =
                        RES ? tc_smem(bres + (size_t)kt * Md::parts * Md::tileB)
                            : base + Md::parts * Md::tileA;
#pragma unroll
                    for (int kk = 0; kk < kTcK / Md::kmma; ++kk) {
                        const uint32_t ko = kk * 2 * kTcLBO;   // one MMA's K = two core matrices
                        const uint64_t ahi = tc_desc(base + ko, Md::sbo);
                        const uint64_t bhi = tc_desc(bbase + ko, Md::sbo);
                        tc_mma<TF32>(acc, ahi, bhi, (kt | kk) != 0);
                        if constexpr (!TF32) {
                            const uint64_t alo = tc_desc(base + Md::tileA + ko, Md::sbo);
                            const uint64_t blo = tc_desc(bbase + Md::tileB + ko, Md::sbo);
                            tc_mma<TF32>(acc, ahi, blo, 1u);
                            tc_mma<TF32>(acc, alo, bhi, 1u);
                        }
                    }
                    tc_commit(&freed[s]);
                }
                if (ok) tc_commit(&acc_full[b]);
            }
            if (!ok) s_fail = 1;
            // every MMA this thread issued is complete before the CTA moves on
            tc_commit(&done);
            if (!tc_mbar_wait(&done, 0)) s_fail = 1;
        }
    } else {
        // epilogue, warp w (0-3) owns accumulator lanes (rows) 32w..32w+31: the
        // tile's 128 columns into registers, the accumulator released, then
        // eight 32-row x 16-column FP64 boxes staged in shared memory (128-byte
        // swizzle, two slots) and written by TMA stores; rows and columns past
        // the ends of chi(R) are clipped by the tensor map
        uint8_t *stg = ring + (size_t)S * SB + (size_t)warp * 2 * kTcBox;
        int mt, nt;
        for (int i = 0; tc_tile<RES>(i, ntn, mtiles, mt, nt); ++i) {
            const int b = i & 1, ub = i >> 1;
            int got = 0;
            if (lane == 0) got = tc_mbar_wait_or_fail(&acc_full[b], (uint32_t)(ub & 1), &s_fail);
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) {
                s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint32_t v[4][32];
            const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * kTcN);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, "
                    "%9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, "
                    "%24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                    : "=r"(v[q][0]), "=r"(v[q][1]), "=r"(v[q][2]), "=r"(v[q][3]), "=r"(v[q][4]),
                      "=r"(v[q][5]), "=r"(v[q][6]), "=r"(v[q][7]), "=r"(v[q][8]), "=r"(v[q][9]),
                      "=r"(v[q][10]), "=r"(v[q][11]), "=r"(v[q][12]), "=r"(v[q][13]),
                      "=r"(v[q][14]), "=r"(v[q][15]), "=r"(v[q][16]), "=r"(v[q][17]),
                      "=r"(v[q][18]), "=r"(v[q][19]), "=r"(v[q][20]), "=r"(v[q][21]),
                      "=r"(v[q][22]), "=r"(v[q][23]), "=r"(v[q][24]), "=r"(v[q][25]),
                      "=r"(v[q][26]), "=r"(v[q][27]), "=r"(v[q][28]), "=r"(v[q][29]),
                      "=r"(v[q][30]), "=r"(v[q][31])
                    : "r"(ta + (uint32_t)(q * 32))
                    : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(
                                 tc_smem(&acc_empty[b]))
                             : "memory");
            const int y = mt * kTcM + warp * 32;
            if constexpr (SUMS) {
                // this lane's row: 64 complex bins of the tile against the
                // channel's target, FP64 sums
                // FP32 products and sums over the tile's 64 bins (the
                // accumulator itself is FP32), FP64 across tiles
                float nu = 0.f, dn = 0.f, R = 0.f, Q = 0.f, P = 0.f, Ru = 0.f, Qu = 0.f;
                const float s0 = (float)sums.s0;
                const int b0 = (nt * kTcN) >> 1;
                // the tile's 64 bins {target re, im, weight, in window}, in
                // FP32, staged once per warp in its (here unused) store boxes;
                // a bin off the window carries zeros, so it adds nothing
                float4 *bw = (float4 *)stg;
                __syncwarp();
                for (int j = lane; j < 64; j += 32) {
                    const int bin = b0 + j;
                    float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (bin < sums.nR) {
                        const double w = sums.wgt[bin];
                        if (w != 0.0)
                            f = make_float4((float)sums.tgt[2 * bin], (float)sums.tgt[2 * bin + 1],
                                            (float)w, 1.f);
                    }
                    bw[j] = f;
                }
                __syncwarp();
#pragma unroll
                for (int j = 0; j < 64; ++j) {
                    const float4 f = bw[j];
                    const float mr = __uint_as_float(v[j >> 4][(j & 15) * 2]);
                    const float mi = __uint_as_float(v[j >> 4][(j & 15) * 2 + 1]);
                    const float rr = fmaf(s0, mr, -f.x), ri = fmaf(s0, mi, -f.y);
                    const float mm = fmaf(mr, mr, mi * mi);
                    const float r2 = fmaf(rr, rr, ri * ri), q2 = fmaf(mr, rr, mi * ri);
                    nu = fmaf(mr, f.x, fmaf(mi, f.y, nu));
                    dn = fmaf(f.w, mm, dn);
                    R = fmaf(f.z, r2, R);
                    Q = fmaf(f.z, q2, Q);
                    P = fmaf(f.z, mm, P);
                    Ru = fmaf(f.w, r2, Ru);
                    Qu = fmaf(f.w, q2, Qu);
                }
                const int row = y + lane;
                if (row < rows) {
                    double *o = sums.part + ((long)row * ntn + nt) * kSums;
                    o[0] = nu;
                    o[1] = dn;
                    o[2] = R;
                    o[3] = Q;
                    o[4] = P;
                    o[5] = Ru;
                    o[6] = Qu;
                }
            } else {
#pragma unroll
            for (int g = 0; g < kTcN / 16; ++g) {
                const int x = nt * kTcN + g * 16;             // even: 16-byte aligned
                uint8_t *box = stg + (g & 1) * kTcBox;
                // the slot's previous store has finished reading it
                if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                __syncwarp();
                // row = lane, 128 bytes; 16-byte chunk c at position c ^ (row & 7)
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const double2 d = make_double2((double)__uint_as_float(v[g >> 1][(g & 1) * 16 + 2 * c]),
                                                   (double)__uint_as_float(v[g >> 1][(g & 1) * 16 + 2 * c + 1]));
                    *(double2 *)(box + lane * 128 + ((c ^ (lane & 7)) << 4)) = d;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    if (x < ncol && y < rows)
                        asm volatile(
                            "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], "
                            "[%3];" ::"l"((uint64_t)&tm_out),
                            "r"(x), "r"(y), "r"(tc_smem(box))
                            : "memory");
                    // one group per box, empty for a box past the ends, so that
                    // "all but the last group read" always means the other slot
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                }
            }
            }   // chi(R) boxes
        }
        // the stores are complete before the CTA leaves
        if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
        __syncwarp();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0 && s_fail) atomicOr(err, CHX_DEVERR_INDEX);
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

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link against the driver library)
typedef CUresult (*TcEncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                               const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                               const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                               CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static TcEncodeFn tc_encode_fn() {
    static TcEncodeFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000,
                                             cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (TcEncodeFn)p;
    }
    return fn;
}

// the contraction as a programmatic dependent of the split: its prologue
// (barriers, tensor memory) overlaps the split's tail, its loads wait for the
// split's end
template <bool TF32, bool RES, bool SUMS>
static cudaError_t tc_launch(int grid, size_t smem, cudaStream_t st, const uint8_t *ahi,
                             const uint8_t *al, int rows, const uint8_t *bhi, const uint8_t *bl,
                             int nkt, int ncol, int ntn, int mtiles, const CUtensorMap &tm,
                             const TcSums &sums, int *err) {
    cudaError_t e = cudaFuncSetAttribute(k_ft_tc<TF32, RES, SUMS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kTcThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_ft_tc<TF32, RES, SUMS>, ahi, al, rows, bhi, bl, nkt, ncol,
                              ntn, mtiles, tm, sums, err);
}

// rows x ntn partial window sums after the operand scratch (the fused form)
static size_t tc_sums_bytes(int rows, int nR) {
    const int ntn = (2 * nR + kTcN - 1) / kTcN;
    return ((size_t)rows * ntn * kSums * sizeof(double) + 255) / 256 * 256;
}

// sum q of row r of out = the sum over column tiles (in order) of its
// partials; one thread per (row, sum)
__global__ void k_tc_sums_reduce(const double *__restrict__ part, int rows, int ntn,
                                 double *__restrict__ out) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)rows * kSums) return;
    const long r = i / kSums;
    const int q = (int)(i - r * kSums);
    double a = 0.0;
    for (int t = 0; t < ntn; ++t) a += part[(r * ntn + t) * kSums + q];
    out[i] = a;
}

// out: chi(R) (sums NULL), or with sums the (rows, 4) window sums
template <bool TF32>
static int ft_batch_tc_mode(const double *chi, int rows, int nk, const double *basis, int nR,
                            double *out, void *scratch, int64_t scratch_bytes, cudaStream_t st,
                            const TcSums *sums = nullptr) {
    typedef TcMode<TF32> Md;
    const TcPlan p = tc_plan(rows, nk, nR, TF32);
    const size_t need = p.total + (sums ? tc_sums_bytes(rows, nR) : 0);
    CHX_REQUIRE(scratch && scratch_bytes >= (int64_t)need,
                "ft_batch: the tensor-core path needs %zu bytes of scratch", need);
    CHX_REQUIRE(((uintptr_t)scratch & 255) == 0, "ft_batch: scratch must be 256-byte aligned");
    CHX_REQUIRE(((uintptr_t)out & 15) == 0,
                "ft_batch: precisions 2 and 3 need out 16-byte aligned");
    const int ncol = 2 * nR;
    // chi(R) (rows x ncol FP64, rows ncol * 8 bytes apart) as the TMA store
    // target, in boxes of 32 rows x 16 columns, 128-byte swizzle (not used by
    // the fused form, which writes sums)
    CUtensorMap tm;
    memset(&tm, 0, sizeof(tm));
    if (!sums) {
        const TcEncodeFn enc = tc_encode_fn();
        CHX_REQUIRE(enc != nullptr, "ft_batch: cuTensorMapEncodeTiled is not available");
        const cuuint64_t gdim[2] = {(cuuint64_t)ncol, (cuuint64_t)rows};
        const cuuint64_t gstride[1] = {(cuuint64_t)ncol * sizeof(double)};
        const cuuint32_t box[2] = {16, 32}, estr[2] = {1, 1};
        const CUresult cr = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void *)out, gdim,
                                gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        CHX_REQUIRE(cr == CUDA_SUCCESS, "ft_batch: chi(R) tensor map refused (CUresult %d)",
                    (int)cr);
    }
    int dev = 0, nsm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "ft_batch device query");

    uint8_t *base = (uint8_t *)scratch;
    int *err = (int *)base;
    const int parts = TF32 ? 1 : 2;
    uint8_t *bhi = base + 256, *bl = bhi + p.b_bytes;
    uint8_t *ahi = base + 256 + parts * p.b_bytes, *al = ahi + p.a_bytes;
    // both operands split by one launch: the basis (its columns are the rows
    // of B) in the first blocks, chi in the rest
    const TcSplitJob jb = {basis, ncol, nk, p.Np, 1, ncol, bhi, bl};
    const TcSplitJob ja = {chi, rows, nk, p.Mp, nk, 1, ahi, al};
    const long nb = (long)p.Np * p.Kp / 8, na = (long)p.Mp * p.Kp / 8;
    const int gb = (int)std::min<long>((nb + 255) / 256, 592);
    const int ga = (int)std::min<long>((na + 255) / 256, 1184);
    k_tc_split<TF32><<<gb + ga, 256, 0, st>>>(jb, ja, p.Kp, gb, err);
    CHX_CHECK_LAUNCH("ft_batch split");

    // persistent: one CTA per SM; the basis tile stays resident when it fits
    // and every column tile has a CTA of its own
    const int ntn = p.Np / kTcN, mtiles = p.Mp / kTcM, nkt = p.Kp / kTcK;
    const int grid = std::min(ntn * mtiles, nsm);
    const bool res = p.Kp <= kTcResKp && ntn <= grid;
    const size_t smem = Md::smem(res, nkt);
    if (sums) {
        TcSums sm = *sums;
        sm.part = (double *)(base + p.total);
        e = res ? tc_launch<TF32, true, true>(grid, smem, st, ahi, al, rows, bhi, bl, nkt, ncol,
                                              ntn, mtiles, tm, sm, err)
                : tc_launch<TF32, false, true>(grid, smem, st, ahi, al, rows, bhi, bl, nkt, ncol,
                                               ntn, mtiles, tm, sm, err);
        if (e != cudaSuccess) return cuda_fail(e, "ft_sums tc launch");
        CHX_CHECK_LAUNCH("ft_sums tc");
        k_tc_sums_reduce<<<(unsigned)(((long)rows * kSums + 255) / 256), 256, 0, st>>>(
            sm.part, rows, ntn, out);
        CHX_CHECK_LAUNCH("ft_sums reduce");
        return CHX_OK;
    }
    const TcSums none = {nullptr, nullptr, nullptr, 0, 1.0};
    e = res ? tc_launch<TF32, true, false>(grid, smem, st, ahi, al, rows, bhi, bl, nkt, ncol, ntn,
                                           mtiles, tm, none, err)
            : tc_launch<TF32, false, false>(grid, smem, st, ahi, al, rows, bhi, bl, nkt, ncol,
                                            ntn, mtiles, tm, none, err);
    if (e != cudaSuccess) return cuda_fail(e, "ft_batch tc launch");
    CHX_CHECK_LAUNCH("ft_batch tc");
    return CHX_OK;
}

int64_t ft_sums_tc_scratch(int rows, int nk, int nR, bool tf32) {
    return (int64_t)(tc_plan(rows, nk, nR, tf32).total + tc_sums_bytes(rows, nR));
}

int ft_sums_tc(const double *chi, int rows, int nk, const double *basis, int nR,
               const double *target, const double *weight, double s0, double *out4,
               void *scratch, int64_t scratch_bytes, cudaStream_t st, bool tf32) {
    const TcSums sums = {target, weight, nullptr, nR, s0};
    return tf32 ? ft_batch_tc_mode<true>(chi, rows, nk, basis, nR, out4, scratch, scratch_bytes,
                                         st, &sums)
                : ft_batch_tc_mode<false>(chi, rows, nk, basis, nR, out4, scratch, scratch_bytes,
                                          st, &sums);
}

int ft_batch_tc(const double *chi, int rows, int nk, const double *basis, int nR, double *out,
                void *scratch, int64_t scratch_bytes, cudaStream_t st, bool tf32) {
    return tf32 ? ft_batch_tc_mode<true>(chi, rows, nk, basis, nR, out, scratch, scratch_bytes, st)
                : ft_batch_tc_mode<false>(chi, rows, nk, basis, nR, out, scratch, scratch_bytes,
                                          st);
}

}  // namespace chx
