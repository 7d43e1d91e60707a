// chx_api.cu -- error reporting and the reference-kernel entry points.
//
// The eight kernels of the reference module (exafs_gpu/kernels.py) are given
// the same arguments and meaning here, so that a caller holding the
// reference's argument tuples can launch them unchanged. The elementwise ones
// are one thread per element, as they must be; chi_forward and chi_delta are
// organised for B200 instead of one block per (k, configuration):
//   chi_forward  one CTA per (chunk of 1024 pairs, configuration); the chunk's
//                pair records are staged in shared memory once and every thread
//                owns one k point, so a block needs no reduction tree and the
//                per-k tables are read once per chunk, not once per pair.
//   chi_delta    one CTA per replica; thread per k over the affected list.
#include <stdarg.h>
#include <stddef.h>
#include <string.h>
#include "chx_device.cuh"

namespace chx {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char *what) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return CHX_ERR_CUDA;
}

// --------------------------------------------------------------- geometry
__global__ void k_compute_r(const double *__restrict__ pos, const int *__restrict__ iidx,
                            const int *__restrict__ jidx, const double *__restrict__ shift,
                            double *__restrict__ r, double *__restrict__ evec, int npairs,
                            int natoms, int nconf) {
    long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long)npairs * nconf) return;
    int ic = (int)(tid / npairs), p = (int)(tid % npairs);
    int i = iidx[p], j = jidx[p];
    const double *pi = pos + ((long)ic * natoms + i) * 3;
    const double *pj = pos + ((long)ic * natoms + j) * 3;
    double dx = pj[0] + shift[3 * p + 0] - pi[0];
    double dy = pj[1] + shift[3 * p + 1] - pi[1];
    double dz = pj[2] + shift[3 * p + 2] - pi[2];
    double rr = sqrt(dx * dx + dy * dy + dz * dz);
    r[tid] = rr;
    if (evec) {
        double inv = 1.0 / rr;
        evec[3 * tid + 0] = dx * inv;
        evec[3 * tid + 1] = dy * inv;
        evec[3 * tid + 2] = dz * inv;
    }
}

__global__ void k_build_ptype(const int *__restrict__ species, const int *__restrict__ iidx,
                              const int *__restrict__ jidx, int *__restrict__ ptype, int npairs,
                              int natoms, int nconf, int nsp) {
    long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long)npairs * nconf) return;
    int ic = (int)(tid / npairs), p = (int)(tid % npairs);
    ptype[tid] = species[(long)ic * natoms + iidx[p]] * nsp + species[(long)ic * natoms + jidx[p]];
}

constexpr int kFwdChunk = 1024;

template <int NSP>
__global__ void __launch_bounds__(256) k_chi_forward(
    const double *__restrict__ r, const int *__restrict__ ptype, const int *__restrict__ shell,
    const double *__restrict__ sig2, const double *__restrict__ ftab,
    const double *__restrict__ dtab, const double *__restrict__ lamtab,
    const double *__restrict__ ktab, const double *__restrict__ drtab,
    const double *__restrict__ c3tab, const double *__restrict__ s2tab, double *__restrict__ chi,
    int npairs, int nk, int nconf, double s02) {
    __shared__ double s_r[kFwdChunk], s_s2[kFwdChunk];
    __shared__ int s_t[kFwdChunk], s_sh[kFwdChunk];
    int ic = blockIdx.y;
    int p0 = blockIdx.x * kFwdChunk;
    int n = min(kFwdChunk, npairs - p0);
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        long g = (long)ic * npairs + p0 + q;
        s_r[q] = r[g];
        s_t[q] = ptype[g];
        s_sh[q] = shell[p0 + q];
        s_s2[q] = sig2[p0 + q];
    }
    __syncthreads();
    for (int ik = threadIdx.x; ik < nk; ik += blockDim.x) {
        KPoint kp{ktab[ik], lamtab[ik]};
        double acc[NSP];
#pragma unroll
        for (int s = 0; s < NSP; ++s) acc[s] = 0.0;
        for (int q = 0; q < n; ++q) {
            int t = s_t[q];
            double v = term64(s_r[q], t, s_sh[q], s_s2[q], ik, nk, NSP, kp, ftab, dtab, drtab,
                              c3tab, s2tab, s02);
            add_by_species<NSP>(acc, t / NSP, v);
        }
#pragma unroll
        for (int s = 0; s < NSP; ++s) atomicAdd(&chi[((long)ic * NSP + s) * nk + ik], acc[s]);
    }
}

template <int NSP>
__global__ void __launch_bounds__(256) k_chi_delta(
    const double *__restrict__ r_old, const int *__restrict__ pt_old,
    const int *__restrict__ shell, const int *__restrict__ aff, const double *__restrict__ r_new,
    const int *__restrict__ pt_new, const double *__restrict__ sig2,
    const double *__restrict__ ftab, const double *__restrict__ dtab,
    const double *__restrict__ lamtab, const double *__restrict__ ktab,
    const double *__restrict__ drtab, const double *__restrict__ c3tab,
    const double *__restrict__ s2tab, double *__restrict__ dchi, int npairs, int nk, int nrep,
    int maxaff, double s02) {
    extern __shared__ double sm_delta[];
    double *s_rn = sm_delta, *s_ro = s_rn + maxaff, *s_s2 = s_ro + maxaff;
    int *s_tn = (int *)(s_s2 + maxaff), *s_to = s_tn + maxaff, *s_sh = s_to + maxaff;
    int ic = blockIdx.x;
    for (int q = threadIdx.x; q < maxaff; q += blockDim.x) {
        int p = aff[(long)ic * maxaff + q];
        if (p < 0) {
            s_sh[q] = -1;
            continue;
        }
        s_rn[q] = r_new[(long)ic * maxaff + q];
        s_tn[q] = pt_new[(long)ic * maxaff + q];
        s_ro[q] = r_old[(long)ic * npairs + p];
        s_to[q] = pt_old[(long)ic * npairs + p];
        s_sh[q] = shell[p];
        s_s2[q] = sig2[p];
    }
    __syncthreads();
    for (int ik = threadIdx.x; ik < nk; ik += blockDim.x) {
        KPoint kp{ktab[ik], lamtab[ik]};
        double acc[NSP];
#pragma unroll
        for (int s = 0; s < NSP; ++s) acc[s] = 0.0;
        for (int q = 0; q < maxaff; ++q) {
            int sh = s_sh[q];
            if (sh < 0) continue;
            int t = s_tn[q];
            add_by_species<NSP>(acc, t / NSP,
                                term64(s_rn[q], t, sh, s_s2[q], ik, nk, NSP, kp, ftab, dtab,
                                       drtab, c3tab, s2tab, s02));
            t = s_to[q];
            add_by_species<NSP>(acc, t / NSP,
                                -term64(s_ro[q], t, sh, s_s2[q], ik, nk, NSP, kp, ftab, dtab,
                                        drtab, c3tab, s2tab, s02));
        }
#pragma unroll
        for (int s = 0; s < NSP; ++s) dchi[((long)ic * NSP + s) * nk + ik] = acc[s];
    }
}

__global__ void k_commit_move(const int *__restrict__ aff, const double *__restrict__ r_new,
                              const int *__restrict__ pt_new, const uint8_t *__restrict__ accept,
                              double *__restrict__ r_old, int *__restrict__ pt_old, int npairs,
                              int nrep, int maxaff) {
    long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long)maxaff * nrep) return;
    int ic = (int)(tid / maxaff);
    if (!accept[ic]) return;
    int p = aff[tid];
    if (p < 0) return;
    r_old[(long)ic * npairs + p] = r_new[tid];
    pt_old[(long)ic * npairs + p] = pt_new[tid];
}

__global__ void k_propose_select(const int *__restrict__ species, const double *__restrict__ pos,
                                 const double *__restrict__ ideal, int *a_out, int *b_out,
                                 int *newsa, int *newsb, double *newpa, uint8_t *isswap,
                                 int natoms, int nrep, uint64_t seed, uint64_t stepc,
                                 double swap_frac, double disp_sigma, double max_disp) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nrep) return;
    const int *S = species + (long)c * natoms;
    const double *P = pos + (long)c * natoms * 3;
    const double *Id = ideal + (long)c * natoms * 3;
    Proposal pr = propose_one([S](int i) { return S[i]; }, P, Id, natoms, seed, stepc, c,
                              swap_frac, disp_sigma, max_disp);
    isswap[c] = (uint8_t)pr.swap;
    a_out[c] = pr.a;
    b_out[c] = pr.b;
    newsa[c] = pr.nsa;
    newsb[c] = pr.nsb;
    newpa[3 * c] = pr.np[0];
    newpa[3 * c + 1] = pr.np[1];
    newpa[3 * c + 2] = pr.np[2];
}

__global__ void k_propose_build(const int *__restrict__ species, const double *__restrict__ pos,
                                const int *__restrict__ nbr, const int *__restrict__ rev,
                                const int *__restrict__ iidx, const int *__restrict__ jidx,
                                const double *__restrict__ shift, const int *__restrict__ a_in,
                                const int *__restrict__ b_in, const int *__restrict__ newsa,
                                const int *__restrict__ newsb, const double *__restrict__ newpa,
                                int *__restrict__ aff, double *__restrict__ r_new,
                                int *__restrict__ pt_new, int natoms, int ncoord, int npairs,
                                int nrep, int maxaff, int nsp) {
    long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long)maxaff * nrep) return;
    int c = (int)(tid / maxaff), q = (int)(tid % maxaff);
    int a = a_in[c], b = b_in[c];
    int blk = q / ncoord, o = q % ncoord;
    int p;
    if (blk == 0) p = nbr[(long)a * ncoord + o];
    else if (blk == 1) p = rev[nbr[(long)a * ncoord + o]];
    else if (blk == 2) p = nbr[(long)b * ncoord + o];
    else p = rev[nbr[(long)b * ncoord + o]];
    if (blk >= 2) {
        if (b == a) p = -1;
        else if (((blk == 2) ? jidx[p] : iidx[p]) == a) p = -1;
    }
    aff[tid] = p;
    if (p < 0) {
        r_new[tid] = 0.0;
        pt_new[tid] = 0;
        return;
    }
    int i = iidx[p], j = jidx[p];
    const double *P = pos + (long)c * natoms * 3;
    const double *NP = newpa + 3 * c;
    const double *pi = (i == a) ? NP : P + 3 * (long)i;
    const double *pj = (j == a) ? NP : P + 3 * (long)j;
    double dx = pj[0] + shift[3 * p + 0] - pi[0];
    double dy = pj[1] + shift[3 * p + 1] - pi[1];
    double dz = pj[2] + shift[3 * p + 2] - pi[2];
    r_new[tid] = sqrt(dx * dx + dy * dy + dz * dz);
    const int *S = species + (long)c * natoms;
    int si = (i == a) ? newsa[c] : ((i == b) ? newsb[c] : S[i]);
    int sj = (j == a) ? newsa[c] : ((j == b) ? newsb[c] : S[j]);
    pt_new[tid] = si * nsp + sj;
}

__global__ void k_commit_state(const uint8_t *__restrict__ accept, const int *__restrict__ a_in,
                               const int *__restrict__ b_in, const int *__restrict__ newsa,
                               const int *__restrict__ newsb, const double *__restrict__ newpa,
                               const uint8_t *__restrict__ isswap, int *__restrict__ species,
                               double *__restrict__ pos, int natoms, int nrep) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nrep || !accept[c]) return;
    int a = a_in[c], b = b_in[c];
    species[(long)c * natoms + a] = newsa[c];
    species[(long)c * natoms + b] = newsb[c];
    if (!isswap[c]) {
        double *P = pos + ((long)c * natoms + a) * 3;
        P[0] = newpa[3 * c];
        P[1] = newpa[3 * c + 1];
        P[2] = newpa[3 * c + 2];
    }
}

static inline unsigned grid1(long n, int tpb = 256) { return (unsigned)((n + tpb - 1) / tpb); }

}  // namespace chx

using namespace chx;

extern "C" {

// Pair-type counts over a subset of pairs, one CTA per configuration:
// counts[c][a * nsp + b] = #{q : species[c][pi[q]] = a, species[c][pj[q]] = b}.
// These are the statistics of the Warren-Cowley parameters
// (exafs_gpu/lattice.py:167-185): alpha_AB = 1 - (n_AB / n_A) / c_B.
__global__ void __launch_bounds__(256) k_pair_counts(const int *__restrict__ species, int natoms,
                                                     const int *__restrict__ pi,
                                                     const int *__restrict__ pj, int npair,
                                                     int nsp, int *__restrict__ counts,
                                                     int *__restrict__ err) {
    __shared__ int s_h[64];
    const int c = blockIdx.x, nn = nsp * nsp;
    for (int q = threadIdx.x; q < nn; q += blockDim.x) s_h[q] = 0;
    __syncthreads();
    const int *S = species + (long)c * natoms;
    for (int q = threadIdx.x; q < npair; q += blockDim.x) {
        const int i = pi[q], j = pj[q];
        if ((unsigned)i >= (unsigned)natoms || (unsigned)j >= (unsigned)natoms) {
            atomicOr(err, CHX_DEVERR_INDEX);
            continue;
        }
        const int a = S[i], b = S[j];
        if ((unsigned)a >= (unsigned)nsp || (unsigned)b >= (unsigned)nsp) {
            atomicOr(err, CHX_DEVERR_INDEX);
            continue;
        }
        atomicAdd(&s_h[a * nsp + b], 1);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nn; q += blockDim.x) counts[(long)c * nn + q] = s_h[q];
}

int chx_version(void) { return 1000; }

int64_t chx_struct_size(int which) {
    switch (which) {
        case 0: return (int64_t)sizeof(chx_pairs_t);
        case 1: return (int64_t)sizeof(chx_ladder_t);
        case 2: return (int64_t)offsetof(chx_ladder_t, exch_acc);
        case 3: return (int64_t)offsetof(chx_ladder_t, seed);
        case 4: return (int64_t)sizeof(chx_mlp_t);
        case 5: return (int64_t)offsetof(chx_ladder_t, log_cap);
        case 6: return (int64_t)sizeof(chx_shell_t);
        case 7: return (int64_t)sizeof(chx_path_t);
        default: return -1;
    }
}

int chx_last_error(char *buf, int n) {
    if (!buf || n <= 0) return CHX_ERR_ARG;
    strncpy(buf, g_err, (size_t)n - 1);
    buf[n - 1] = 0;
    return CHX_OK;
}

int chx_compute_r(const double *pos, const int *iidx, const int *jidx, const double *shift,
                  double *r, double *evec, int npairs, int natoms, int nconf, void *stream) {
    CHX_REQUIRE(pos && iidx && jidx && shift && r && npairs > 0 && nconf > 0,
                "compute_r: bad arguments");
    long n = (long)npairs * nconf;
    k_compute_r<<<grid1(n), 256, 0, as_stream(stream)>>>(pos, iidx, jidx, shift, r, evec, npairs,
                                                         natoms, nconf);
    CHX_CHECK_LAUNCH("compute_r");
    return CHX_OK;
}

int chx_build_ptype(const int *species, const int *iidx, const int *jidx, int *ptype,
                    int npairs, int natoms, int nconf, int nsp, void *stream) {
    CHX_REQUIRE(species && iidx && jidx && ptype && npairs > 0 && nconf > 0 && nsp >= 2,
                "build_ptype: bad arguments");
    long n = (long)npairs * nconf;
    k_build_ptype<<<grid1(n), 256, 0, as_stream(stream)>>>(species, iidx, jidx, ptype, npairs,
                                                           natoms, nconf, nsp);
    CHX_CHECK_LAUNCH("build_ptype");
    return CHX_OK;
}

int chx_chi_forward(const double *r, const int *ptype, const int *shell, const double *sig2,
                    const double *ftab, const double *dtab, const double *lamtab,
                    const double *ktab, const double *drtab, const double *c3tab,
                    const double *s2tab, double *chi, int npairs, int nk, int nconf, double s02,
                    int nsp, void *stream) {
    CHX_REQUIRE(r && ptype && shell && sig2 && ftab && dtab && lamtab && ktab && drtab &&
                    c3tab && s2tab && chi && npairs > 0 && nk > 0 && nconf > 0,
                "chi_forward: bad arguments");
    cudaStream_t st = as_stream(stream);
    cudaError_t e = cudaMemsetAsync(chi, 0, sizeof(double) * (size_t)nconf * nsp * nk, st);
    if (e != cudaSuccess) return cuda_fail(e, "chi_forward memset");
    dim3 grid((npairs + kFwdChunk - 1) / kFwdChunk, nconf);
#define CHX_FWD(N)                                                                          \
    k_chi_forward<N><<<grid, 256, 0, st>>>(r, ptype, shell, sig2, ftab, dtab, lamtab, ktab,  \
                                           drtab, c3tab, s2tab, chi, npairs, nk, nconf, s02)
    switch (nsp) {
        case 2: CHX_FWD(2); break;
        case 3: CHX_FWD(3); break;
        case 4: CHX_FWD(4); break;
        default: set_error("chi_forward: nsp %d not built (2..4)", nsp); return CHX_ERR_UNSUPPORTED;
    }
#undef CHX_FWD
    CHX_CHECK_LAUNCH("chi_forward");
    return CHX_OK;
}

int chx_chi_delta(const double *r_old, const int *pt_old, const int *shell, const int *aff,
                  const double *r_new, const int *pt_new, const double *sig2,
                  const double *ftab, const double *dtab, const double *lamtab,
                  const double *ktab, const double *drtab, const double *c3tab,
                  const double *s2tab, double *dchi, int npairs, int nk, int nrep, int maxaff,
                  double s02, int nsp, void *stream) {
    CHX_REQUIRE(r_old && pt_old && shell && aff && r_new && pt_new && dchi && nrep > 0 &&
                    maxaff > 0 && maxaff <= 4096,
                "chi_delta: bad arguments");
    size_t smem = (size_t)maxaff * (3 * sizeof(double) + 3 * sizeof(int));
    cudaStream_t st = as_stream(stream);
#define CHX_DEL(N)                                                                            \
    do {                                                                                      \
        if (smem > 48 * 1024)                                                                 \
            cudaFuncSetAttribute(k_chi_delta<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                 (int)smem);                                                  \
        k_chi_delta<N><<<nrep, 256, smem, st>>>(r_old, pt_old, shell, aff, r_new, pt_new, sig2, \
                                                ftab, dtab, lamtab, ktab, drtab, c3tab, s2tab, \
                                                dchi, npairs, nk, nrep, maxaff, s02);          \
    } while (0)
    switch (nsp) {
        case 2: CHX_DEL(2); break;
        case 3: CHX_DEL(3); break;
        case 4: CHX_DEL(4); break;
        default: set_error("chi_delta: nsp %d not built (2..4)", nsp); return CHX_ERR_UNSUPPORTED;
    }
#undef CHX_DEL
    CHX_CHECK_LAUNCH("chi_delta");
    return CHX_OK;
}

int chx_commit_move(const int *aff, const double *r_new, const int *pt_new,
                    const uint8_t *accept, double *r_old, int *pt_old, int npairs, int nrep,
                    int maxaff, void *stream) {
    CHX_REQUIRE(aff && r_new && pt_new && accept && r_old && pt_old, "commit_move: bad arguments");
    k_commit_move<<<grid1((long)maxaff * nrep), 256, 0, as_stream(stream)>>>(
        aff, r_new, pt_new, accept, r_old, pt_old, npairs, nrep, maxaff);
    CHX_CHECK_LAUNCH("commit_move");
    return CHX_OK;
}

int chx_propose_select(const int *species, const double *pos, const double *ideal, int *a_out,
                       int *b_out, int *newsa, int *newsb, double *newpa, uint8_t *isswap,
                       int natoms, int nrep, uint64_t seed, uint64_t stepc, double swap_frac,
                       double disp_sigma, double max_disp, void *stream) {
    CHX_REQUIRE(species && pos && ideal && a_out && b_out && newsa && newsb && newpa && isswap &&
                    natoms > 0 && nrep > 0,
                "propose_select: bad arguments");
    k_propose_select<<<grid1(nrep), 256, 0, as_stream(stream)>>>(
        species, pos, ideal, a_out, b_out, newsa, newsb, newpa, isswap, natoms, nrep, seed, stepc,
        swap_frac, disp_sigma, max_disp);
    CHX_CHECK_LAUNCH("propose_select");
    return CHX_OK;
}

int chx_propose_build(const int *species, const double *pos, const int *nbr, const int *rev,
                      const int *iidx, const int *jidx, const double *shift, const int *a_in,
                      const int *b_in, const int *newsa, const int *newsb, const double *newpa,
                      int *aff, double *r_new, int *pt_new, int natoms, int ncoord, int npairs,
                      int nrep, int maxaff, int nsp, void *stream) {
    CHX_REQUIRE(species && pos && nbr && rev && iidx && jidx && shift && aff && r_new &&
                    pt_new && maxaff == 4 * ncoord,
                "propose_build: bad arguments (maxaff must be 4*ncoord)");
    k_propose_build<<<grid1((long)maxaff * nrep), 256, 0, as_stream(stream)>>>(
        species, pos, nbr, rev, iidx, jidx, shift, a_in, b_in, newsa, newsb, newpa, aff, r_new,
        pt_new, natoms, ncoord, npairs, nrep, maxaff, nsp);
    CHX_CHECK_LAUNCH("propose_build");
    return CHX_OK;
}

int chx_commit_state(const uint8_t *accept, const int *a_in, const int *b_in,
                     const int *newsa, const int *newsb, const double *newpa,
                     const uint8_t *isswap, int *species, double *pos, int natoms, int nrep,
                     void *stream) {
    CHX_REQUIRE(accept && a_in && b_in && newsa && newsb && newpa && isswap && species && pos,
                "commit_state: bad arguments");
    k_commit_state<<<grid1(nrep), 256, 0, as_stream(stream)>>>(accept, a_in, b_in, newsa, newsb,
                                                               newpa, isswap, species, pos,
                                                               natoms, nrep);
    CHX_CHECK_LAUNCH("commit_state");
    return CHX_OK;
}

int chx_pair_counts(const int *species, int nconf, int natoms, const int *pi, const int *pj,
                    int npair, int nsp, int *counts, int *d_err, void *stream) {
    CHX_REQUIRE(species && pi && pj && counts && d_err && nconf > 0 && natoms > 0 && npair > 0 &&
                    nsp >= 1 && nsp <= 8,
                "pair_counts: bad arguments (nsp 1..8)");
    k_pair_counts<<<nconf, 256, 0, as_stream(stream)>>>(species, natoms, pi, pj, npair, nsp,
                                                        counts, d_err);
    CHX_CHECK_LAUNCH("pair_counts");
    return CHX_OK;
}

}  // extern "C"
