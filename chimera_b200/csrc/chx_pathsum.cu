// chx_pathsum.cu -- full single-scattering path sum (A1) and exact
// supercell multiple-scattering counts (A2).
//
// Path sum, three launches on one stream:
//   k_pair_records  one thread per (configuration, pair): r from positions
//                   (exafs_gpu/kernels.py:53-78), pair type from species
//                   (kernels.py:81-96), folded with the per-(shell, type)
//                   offsets into a 32-byte record {r_eff, sigma^2, C3, 1/r_eff^2, t}.
//   k_pathsum       one CTA per (run of pair chunks, configuration); a single
//                   elected thread streams 256-record chunks into a
//                   double-buffered shared-memory ring with cp.async.bulk
//                   (TMA bulk copies, no multicast) completing on mbarriers;
//                   every thread owns one k point and accumulates the chunk's
//                   terms for its k in registers (k-vectorised per warp: the
//                   32 lanes of a warp evaluate one path at 32 consecutive k).
//                   Each CTA writes its partial spectrum to scratch.
//   k_reduce_partials  fixed-order sum of the partials: deterministic chi.
//
// Precision (CHX_FP32C): the phase 2 k r_eff + delta - 4/3 k^3 C3 and its
// reduction to [-pi, pi] are FP64, the sine, exponential and amplitude are
// FP32, and every term is accumulated in FP64. CHX_FP64 evaluates the
// reference's FP64 formula unchanged.
#include <algorithm>
#include "chx_device.cuh"

namespace chx {

constexpr int kChunk = 256;        // records per bulk copy (8 KB)
constexpr int kMaxChunksPerCta = 64;
constexpr int kBulkSpin = 1 << 26; // bounded wait on a bulk copy

__global__ void k_pair_records(const double *__restrict__ pos, const int *__restrict__ species,
                               chx_pairs_t P, int nconf, PairRec *__restrict__ rec,
                               int *__restrict__ err) {
    long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long)P.npairs * nconf) return;
    int ic = (int)(tid / P.npairs), p = (int)(tid % P.npairs);
    int i = P.iidx[p], j = P.jidx[p];
    if ((unsigned)i >= (unsigned)P.natoms || (unsigned)j >= (unsigned)P.natoms) {
        atomicOr(err, CHX_DEVERR_INDEX);
        rec[tid] = PairRec{1.0, 0.0, 0.0, 0.0f, -1};
        return;
    }
    int nsp = P.nsp, nn = nsp * nsp;
    const int si = species[(long)ic * P.natoms + i], sj = species[(long)ic * P.natoms + j];
    const int sh = P.shell[p];
    // species and shell index the per-type tables: out of range, the pair is
    // dropped (sentinel record) and the call's error word is set
    if ((unsigned)si >= (unsigned)nsp || (unsigned)sj >= (unsigned)nsp ||
        (unsigned)sh >= (unsigned)P.nshell) {
        atomicOr(err, CHX_DEVERR_INDEX);
        rec[tid] = PairRec{1.0, 0.0, 0.0, 0.0f, -1};
        return;
    }
    const double *pi = pos + ((long)ic * P.natoms + i) * 3;
    const double *pj = pos + ((long)ic * P.natoms + j) * 3;
    double dx = pj[0] + P.shift[3 * p + 0] - pi[0];
    double dy = pj[1] + P.shift[3 * p + 1] - pi[1];
    double dz = pj[2] + P.shift[3 * p + 2] - pi[2];
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    int t = si * nsp + sj;
    double reff = r + P.drtab[sh * nn + t];
    PairRec o;
    o.reff = reff;
    o.s2 = P.sig2[p] + P.s2tab[sh * nn + t];
    o.c3 = P.c3tab[sh];
    o.inv_r2 = (float)(1.0 / (reff * reff));
    o.t = t;
    rec[tid] = o;
}

// ------------------------------------------------------- bulk copy helpers
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// Wait for phase `parity` of the barrier, at most kBulkSpin polls; returns
// false (and the caller records an error) if the copy never completed.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    uint32_t a = smem_addr(bar);
    for (int it = 0; it < kBulkSpin; ++it) {
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

// grid (ncta, nconf); block = nk rounded up to a warp multiple (<= 512)
template <int NSP, int PREC>
__global__ void __launch_bounds__(512) k_pathsum(const PairRec *__restrict__ rec, chx_pairs_t P,
                                                 int chunks_per_cta, double *__restrict__ partial,
                                                 int *__restrict__ err) {
    __shared__ __align__(128) PairRec ring[2][kChunk];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_fail;
    int ic = blockIdx.y;
    int nchunk_total = (P.npairs + kChunk - 1) / kChunk;
    int c0 = blockIdx.x * chunks_per_cta;
    int nch = min(chunks_per_cta, nchunk_total - c0);
    const PairRec *base = rec + (long)ic * P.npairs;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](int ci) {
        int p0 = (c0 + ci) * kChunk;
        int n = min(kChunk, P.npairs - p0);
        uint32_t bytes = (uint32_t)(n * sizeof(PairRec));
        uint64_t *b = &bar[ci & 1];
        // order this CTA's earlier generic-proxy reads of the buffer before
        // the async-proxy write that refills it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(b, bytes);
        bulk_g2s(ring[ci & 1], base + p0, bytes, b);
    };
    if (threadIdx.x == 0 && nch > 0) {
        issue(0);
        if (nch > 1) issue(1);
    }
    int ik = threadIdx.x;
    bool active = ik < P.nk;
    KConst<NSP> kc;
    if (active) load_kconst<NSP>(kc, P.ktab, P.lamtab, P.dtab, P.ftab, P.s02, P.nk, ik);
    double acc[NSP];
#pragma unroll
    for (int s = 0; s < NSP; ++s) acc[s] = 0.0;
    int cfail = -1;   // the chunk whose wait ran out
    for (int ci = 0; ci < nch; ++ci) {
        if (!mbar_wait(&bar[ci & 1], (uint32_t)((ci >> 1) & 1))) s_fail = 1;
        __syncthreads();
        if (s_fail) {
            cfail = ci;
            break;
        }
        int n = min(kChunk, P.npairs - (c0 + ci) * kChunk);
        const PairRec *rr = ring[ci & 1];
        if (active) {
            for (int q = 0; q < n; ++q) {
                PairRec r = rr[q];
                if (r.t < 0) continue;
                add_by_species<NSP>(acc, r.t / NSP, rec_term<NSP, PREC>(r, kc));
            }
        }
        __syncthreads();  // every thread is done with this buffer
        if (threadIdx.x == 0 && ci + 2 < nch) issue(ci + 2);
    }
    if (s_fail) {
        if (threadIdx.x == 0) {
            atomicOr(err, CHX_DEVERR_INDEX);
            // before the CTA's shared memory is released, wait (bounded) for
            // the copies that may still be in flight: the failed chunk and
            // the one issued after it into the other ring slot
            for (int c = cfail; c < min(nch, cfail + 2); ++c)
                (void)mbar_wait(&bar[c & 1], (uint32_t)((c >> 1) & 1));
        }
        return;
    }
    if (active) {
        long o = (((long)ic * gridDim.x + blockIdx.x) * NSP) * P.nk + ik;
#pragma unroll
        for (int s = 0; s < NSP; ++s) partial[o + (long)s * P.nk] = acc[s];
    }
}

// chi[ic][s][k] = sum over CTAs (in order) of partial[ic][cta][s][k]
// A call whose error word is set (an index out of range, or a bulk-copy wait
// that ran out and left partials unwritten) writes NaN to every chi value, so
// the failure shows in the output even where the caller cannot read the word.
__global__ void k_reduce_partials(const double *__restrict__ partial, int ncta, int nsp, int nk,
                                  int nconf, const int *__restrict__ err,
                                  double *__restrict__ chi) {
    long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long per = (long)nsp * nk;
    if (tid >= per * nconf) return;
    if (*(volatile const int *)err != 0) {
        chi[tid] = __longlong_as_double(0x7FF8000000000000LL);
        return;
    }
    int ic = (int)(tid / per);
    long sk = tid % per;
    const double *p = partial + (long)ic * ncta * per + sk;
    double s = 0.0;
    for (int c = 0; c < ncta; ++c) s += p[(long)c * per];
    chi[tid] = s;
}

struct PathsumPlan {
    int chunks_per_cta, ncta, threads;
    size_t rec_bytes, partial_bytes;
};

static PathsumPlan plan_pathsum(const chx_pairs_t *P, int nconf) {
    PathsumPlan pl;
    long nchunk = (P->npairs + kChunk - 1) / kChunk;
    // aim for at least 4 resident CTAs per SM over the whole launch
    long want = (long)kNumSMs * 4;
    long per = (nchunk * nconf + want - 1) / want;
    pl.chunks_per_cta = (int)std::min<long>(kMaxChunksPerCta, std::max<long>(1, per));
    pl.ncta = (int)((nchunk + pl.chunks_per_cta - 1) / pl.chunks_per_cta);
    pl.threads = ((P->nk + 31) / 32) * 32;
    pl.rec_bytes = sizeof(PairRec) * (size_t)P->npairs * nconf;
    pl.partial_bytes = sizeof(double) * (size_t)nconf * pl.ncta * P->nsp * P->nk;
    return pl;
}

// ------------------------------------------------------- multiple scattering
// Entry of one path record {abs | cls << 20, s0, s1, s2} (mslibrary.py:433-434)
__device__ __forceinline__ int ms_entry(const int *S, int4 rc, int nsp, int nblk) {
    int ab = rc.x & 0xFFFFF;
    int e = S[ab] * nblk + (rc.x >> 20);
    int pw = 1;
    if (rc.y >= 0) e += S[rc.y] * pw;
    pw *= nsp;
    if (rc.z >= 0) e += S[rc.z] * pw;
    pw *= nsp;
    if (rc.w >= 0) e += S[rc.w] * pw;
    return e;
}

// grid (ncta, nconf): a shared-memory histogram of entries per CTA
__global__ void __launch_bounds__(256) k_ms_counts(const int *__restrict__ species, int natoms,
                                                   const int4 *__restrict__ paths, long npath,
                                                   int nsp, int nblk, int *__restrict__ counts,
                                                   long per_cta) {
    extern __shared__ int hist[];
    int nent = nsp * nblk;
    int ic = blockIdx.y;
    for (int e = threadIdx.x; e < nent; e += blockDim.x) hist[e] = 0;
    __syncthreads();
    const int *S = species + (long)ic * natoms;
    long p0 = (long)blockIdx.x * per_cta, p1 = min(npath, p0 + per_cta);
    for (long p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
        int4 rc = __ldg(&paths[p]);
        atomicAdd(&hist[ms_entry(S, rc, nsp, nblk)], 1);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nent; e += blockDim.x)
        if (hist[e]) atomicAdd(&counts[(long)ic * nent + e], hist[e]);
}


// one CTA per replica: the change of the entry counts along the paths through
// a and b (the sampler step does the same inline)
__global__ void __launch_bounds__(256) k_ms_delta(const int *__restrict__ species, int natoms,
                                                  const int4 *__restrict__ inc, int M, int nsp,
                                                  int nblk, const int *__restrict__ a_in,
                                                  const int *__restrict__ b_in,
                                                  const int *__restrict__ nsa_in,
                                                  const int *__restrict__ nsb_in,
                                                  int *__restrict__ dC) {
    extern __shared__ int hist[];
    int nent = nsp * nblk, c = blockIdx.x;
    for (int e = threadIdx.x; e < nent; e += blockDim.x) hist[e] = 0;
    __syncthreads();
    const int *S = species + (long)c * natoms;
    int a = a_in[c], b = b_in[c], nsa = nsa_in[c], nsb = nsb_in[c];
    auto sp = [&](int site) { return site == a ? nsa : (site == b ? nsb : S[site]); };
    for (int m = threadIdx.x; m < 2 * M; m += blockDim.x) {
        int half = m >= M;
        if (half && b == a) break;
        int4 rc = __ldg(&inc[(long)(half ? b : a) * M + (m - half * M)]);
        if (rc.x < 0) continue;
        int ab = rc.x & 0xFFFFF;
        if (half && (ab == a || rc.y == a || rc.z == a || rc.w == a)) continue;
        int eo = ms_entry(S, rc, nsp, nblk);
        int en = sp(ab) * nblk + (rc.x >> 20);
        int pw = 1;
        if (rc.y >= 0) en += sp(rc.y) * pw;
        pw *= nsp;
        if (rc.z >= 0) en += sp(rc.z) * pw;
        pw *= nsp;
        if (rc.w >= 0) en += sp(rc.w) * pw;
        if (en != eo) {
            atomicAdd(&hist[en], 1);
            atomicSub(&hist[eo], 1);
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nent; e += blockDim.x) dC[(long)c * nent + e] = hist[e];
}

// chi[ic][a][k] += sum_e counts[ic][a*nblk+e] T[a*nblk+e][k]; grid (nconf, nsp)
__global__ void k_ms_chi_of(const int *__restrict__ counts, const double *__restrict__ T,
                            int nsp, int nblk, int nk, double *__restrict__ chi) {
    int ic = blockIdx.x, a = blockIdx.y;
    const int *C = counts + ((long)ic * nsp + a) * nblk;
    const double *Ta = T + (long)a * nblk * nk;
    for (int ik = threadIdx.x; ik < nk; ik += blockDim.x) {
        double s = 0.0;
        for (int e = 0; e < nblk; ++e) {
            int c = C[e];
            if (c) s += (double)c * Ta[(long)e * nk + ik];
        }
        chi[((long)ic * nsp + a) * nk + ik] += s;
    }
}

}  // namespace chx

using namespace chx;

extern "C" {

int64_t chx_chi_full_scratch_bytes(const chx_pairs_t *P, int nconf) {
    if (!P || nconf <= 0 || P->npairs <= 0) return -1;
    PathsumPlan pl = plan_pathsum(P, nconf);
    // records, partials, one error word, each 256-byte aligned
    return (int64_t)(((pl.rec_bytes + 255) / 256) * 256 + ((pl.partial_bytes + 255) / 256) * 256 +
                     256);
}

int chx_chi_full(const chx_pairs_t *P, const double *pos, const int *species, int nconf,
                 int precision, double *chi, void *scratch, int64_t scratch_bytes,
                 void *stream) {
    CHX_REQUIRE(P && pos && species && chi && nconf > 0 && P->npairs > 0 && P->nk > 0 &&
                    P->nk <= 512 && P->iidx && P->jidx && P->shift && P->shell && P->sig2 &&
                    P->ftab && P->dtab && P->lamtab && P->ktab && P->drtab && P->c3tab &&
                    P->s2tab,
                "chi_full: bad arguments (nk must be 1..512)");
    CHX_REQUIRE(precision == CHX_FP64 || precision == CHX_FP32C, "chi_full: bad precision %d",
                precision);
    int64_t need = chx_chi_full_scratch_bytes(P, nconf);
    if (!scratch || scratch_bytes < need) {
        set_error("chi_full: scratch of %lld bytes needed, %lld given", (long long)need,
                  (long long)scratch_bytes);
        return CHX_ERR_SCRATCH;
    }
    PathsumPlan pl = plan_pathsum(P, nconf);
    char *s = (char *)scratch;
    PairRec *rec = (PairRec *)s;
    s += ((pl.rec_bytes + 255) / 256) * 256;
    double *partial = (double *)s;
    s += ((pl.partial_bytes + 255) / 256) * 256;
    int *err = (int *)s;
    cudaStream_t st = as_stream(stream);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "chi_full memset");
    long n = (long)P->npairs * nconf;
    k_pair_records<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pos, species, *P, nconf, rec, err);
    CHX_CHECK_LAUNCH("chi_full records");
    dim3 grid(pl.ncta, nconf);
#define CHX_PS(N, PR) k_pathsum<N, PR><<<grid, pl.threads, 0, st>>>(rec, *P, pl.chunks_per_cta, partial, err)
    if (precision == CHX_FP64) {
        switch (P->nsp) {
            case 2: CHX_PS(2, CHX_FP64); break;
            case 3: CHX_PS(3, CHX_FP64); break;
            case 4: CHX_PS(4, CHX_FP64); break;
            default: set_error("chi_full: nsp %d not built", P->nsp); return CHX_ERR_UNSUPPORTED;
        }
    } else {
        switch (P->nsp) {
            case 2: CHX_PS(2, CHX_FP32C); break;
            case 3: CHX_PS(3, CHX_FP32C); break;
            case 4: CHX_PS(4, CHX_FP32C); break;
            default: set_error("chi_full: nsp %d not built", P->nsp); return CHX_ERR_UNSUPPORTED;
        }
    }
#undef CHX_PS
    CHX_CHECK_LAUNCH("chi_full pathsum");
    long m = (long)nconf * P->nsp * P->nk;
    k_reduce_partials<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(partial, pl.ncta, P->nsp,
                                                                   P->nk, nconf, err, chi);
    CHX_CHECK_LAUNCH("chi_full reduce");
    return CHX_OK;
}

int chx_ms_counts(const int *species, int nconf, int natoms, const int *paths, int64_t npath,
                  int nsp, int nblk, int *counts, void *stream) {
    CHX_REQUIRE(species && paths && counts && nconf > 0 && npath > 0 && nsp >= 2 &&
                    nblk > 0 && natoms > 0 && natoms < (1 << 20),
                "ms_counts: bad arguments");
    int nent = nsp * nblk;
    size_t smem = sizeof(int) * (size_t)nent;
    CHX_REQUIRE(smem <= 200 * 1024, "ms_counts: %d entries do not fit shared memory", nent);
    cudaStream_t st = as_stream(stream);
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)nconf * nent, st);
    if (e != cudaSuccess) return cuda_fail(e, "ms_counts memset");
    long want = (long)kNumSMs * 4;
    long per_conf = std::max<long>(1, (want + nconf - 1) / nconf);
    long per_cta = std::max<long>(4096, (npath + per_conf - 1) / per_conf);
    int ncta = (int)((npath + per_cta - 1) / per_cta);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_ms_counts, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_ms_counts<<<dim3(ncta, nconf), 256, smem, st>>>(species, natoms, (const int4 *)paths, npath,
                                                      nsp, nblk, counts, per_cta);
    CHX_CHECK_LAUNCH("ms_counts");
    return CHX_OK;
}

int chx_ms_delta(const int *species, int nrep, int natoms, const int *inc, int M, int nsp,
                 int nblk, const int *a, const int *b, const int *nsa, const int *nsb, int *dC,
                 void *stream) {
    CHX_REQUIRE(species && inc && a && b && nsa && nsb && dC && nrep > 0 && M > 0 &&
                    nsp >= 2 && nblk > 0,
                "ms_delta: bad arguments");
    size_t smem = sizeof(int) * (size_t)nsp * nblk;
    CHX_REQUIRE(smem <= 200 * 1024, "ms_delta: entries do not fit shared memory");
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_ms_delta, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_ms_delta<<<nrep, 256, smem, as_stream(stream)>>>(species, natoms, (const int4 *)inc, M,
                                                       nsp, nblk, a, b, nsa, nsb, dC);
    CHX_CHECK_LAUNCH("ms_delta");
    return CHX_OK;
}

int chx_ms_chi_of(const int *counts, const double *T, int nconf, int nsp, int nblk, int nk,
                  double *chi, void *stream) {
    CHX_REQUIRE(counts && T && chi && nconf > 0 && nsp >= 2 && nblk > 0 && nk > 0,
                "ms_chi_of: bad arguments");
    k_ms_chi_of<<<dim3(nconf, nsp), 256, 0, as_stream(stream)>>>(counts, T, nsp, nblk, nk, chi);
    CHX_CHECK_LAUNCH("ms_chi_of");
    return CHX_OK;
}

}  // extern "C"
