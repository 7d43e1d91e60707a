// chx_sampler.cu -- the fused parallel-tempering RMC step (A3-A7), the
// replica exchange (A8) and the ideal-shell term table.
//
// One CTA per replica slot runs `nsteps` consecutive steps of
// methods/method_a_rmc.py (RMCSampler.step, :250-308) for its replica.
// Replicas only interact at replica exchange, so a launch covers the steps
// between two exchanges and the replica's species live in shared memory for
// all of them (one byte per site: species in bits 0-6, "displaced from its
// ideal site" in bit 7). Each step:
//   1. propose: the reference's splitmix64 stream keyed (seed, step, rung),
//      bit-identical (exafs_gpu/kernels.py:362-423);
//   2. the affected directed pairs: both directions of every bond of a, and of
//      b with the pairs through a dropped (kernels.py:425-488); old and new
//      (r, type) of each, r recomputed from the positions when needed;
//   3. delta chi(k) of those pairs (kernels.py:243-325). In CHX_FP32C a pair
//      whose two atoms sit on their ideal sites takes its term from the
//      (shell, pair type) table, so a swap costs a count of type changes
//      instead of transcendentals; displaced pairs and CHX_FP64 evaluate the
//      term directly. The MS paths through a and b are re-counted from their
//      incidence records (chimera/mslibrary.py:466-486) and contracted with
//      the entry table;
//   4. the trial chi, normalised per absorber and shifted by chi_extra, is
//      resampled, windowed and transformed on the fit-window R bins only
//      (exafs_gpu/fourier.py:69-80, chimera/multift.py:58-63): one thread per
//      (bin, half of the taps) accumulates every channel, the twiddle
//      e^{-2 pi i n m / nfft} advanced by complex rotation and re-seeded
//      exactly (sincospi) every 32 taps;
//   5. profiled-scale chi^2 (method_a_rmc.py:190-227), Metropolis with the
//      energy prior (method_a_rmc.py:280-285, 310-320);
//   6. commit of species, position, chi, chi^2, MS counts and best state
//      (kernels.py:328-346, 490-511; method_a_rmc.py:298-307).
// The last CTA to finish advances the step counter, so a sequence of blocks
// is a sequence of identical launches (CUDA-graph capturable).
#include <cuda_bf16.h>
#include "chx_device.cuh"
#include "chx_mlp.cuh"

namespace chx {

constexpr int kStepThreads = 256;
constexpr int kMaxCoord = 256;
constexpr int kReseed = 32;      // taps between exact twiddles in the transform
constexpr int kMaxSplit = 2;     // threads sharing one bin's taps
constexpr int kUndo = 32;        // accepted moves kept after a slot's best point
// MS entry counts below this are resolved from packed words (old entry in
// bits 0-13, new entry in bits 14-27, occurrences of site a in 28-31)
constexpr int kMsPackMax = 1 << 14;
// The near-tie test's model of the FP32 parts of a move's change: each is an
// independent relative rounding of RMS at most eps (a direct record's term:
// FP32 exp, sin of an FP64-reduced phase, amplitude products; an MS row
// rounded from FP64 to FP32, and each FP32 accumulation step of the MS rows:
// 2^-24 / sqrt(3)), summed in quadrature, and the bound taken at kTieSigma
// standard deviations; the (shell, type) rows and the other accumulations of
// the change are FP64 and add nothing
constexpr double kEpsRec = 2e-7;
constexpr double kEpsTab = 3.5e-8;
constexpr double kTieSigma = 6.0;

// Shared-memory carve-up of one step CTA (all offsets 16-byte aligned).
// The near-tie FP64 transforms reuse the span u .. dirv (the resampled rows,
// the transform's output and the direct records, all rebuilt every step).
struct StepSmem {
    size_t u, x, dir, dirv, tr, dchi, hist, dn, list, sp, nb, nbm, cd, chi, total;
    size_t tie;      // bytes the FP64 near-tie buffers need (0: none)
};

// salt of the stage-1 uniforms of delayed acceptance
constexpr uint64_t kDaSalt = 0x6A09E667F3BCC909ULL;

template <typename T>
__host__ __device__ static inline size_t al16(size_t n) { return ((n * sizeof(T)) + 15) / 16 * 16; }

static StepSmem step_smem(const chx_ladder_t &L, int precision) {
    StepSmem s;
    bool f64 = precision == CHX_FP64;
    size_t o = 0;
    int maxaff = 4 * L.ncoord;
    int nent = L.ms_nblk ? L.nsp * L.ms_nblk : 0;
    int ndn = L.nshell * L.nsp * L.nsp;
    // resampled rows, channel stride padded to even (channel pairs of the DFT)
    const size_t nchp = (size_t)L.nchan + (L.nchan & 1);
    s.u = o; o += f64 ? al16<double>(nchp * L.ncoef) : al16<float>(nchp * L.ncoef);
    if (!f64 && L.xr && L.ft_frag) {
        // the change's BF16 hi/lo operands of the tensor-core transform,
        // channel-major with a padded row stride (tc_row_stride)
        const size_t need = al16<uint16_t>((size_t)2 * ((L.nchan + 7) / 8 * 8) *
                                           (L.ft_kt * 16 + 8));
        if (o - s.u < need) o = s.u + need;
    }
    size_t xs = f64 ? al16<double2>((size_t)kMaxSplit * L.nchan * L.nwin)
                    : al16<float2>((size_t)kMaxSplit * L.nchan * L.nwin);
    // the surrogate's scratch (partial sums of every warp + one activation
    // row, H <= 256) shares the transform's region: they are used in turn
    if (L.mlp) xs = std::max(xs, al16<float>((size_t)(kStepThreads / 32 + 1) * 256));
    s.x = o; o += xs;
    s.dir = o; o += al16<PairRec>((size_t)2 * maxaff);
    s.dirv = o; o += al16<int>((size_t)2 * maxaff);
    // FP64 resampled rows and one split of the FP64 window transform
    s.tie = (!f64 && L.xr)
                ? al16<double>(nchp * L.ncoef) + al16<double2>((size_t)L.nchan * L.nwin)
                : 0;
    if (o - s.u < s.tie) o = s.u + s.tie;   // the span must hold them
    s.tr = o; o += al16<double>((size_t)L.nsp * L.nk);
    s.dchi = o; o += al16<double>((size_t)L.nsp * L.nk);
    s.hist = o; o += al16<int>((size_t)std::max(nent, 1));
    s.dn = o; o += al16<int>((size_t)std::max(ndn, 1));
    s.list = o; o += al16<int>((size_t)(2 * maxaff + 2 * ndn + 2 * nent + 64));
    s.sp = o; o += al16<uint8_t>((size_t)L.natoms);
    s.nb = o; o += al16<uint16_t>((size_t)2 * (std::max(L.ms_D, 1) + 2));
    // the neighbourhood words of both sites premultiplied per template
    // position (kMsPackMax), 4 x (D + 2) each
    s.nbm = o; o += al16<uint32_t>((size_t)8 * (std::max(L.ms_D, 1) + 2));
    s.cd = o; o += al16<uint8_t>((size_t)((L.mlp || L.log_cap > 0) ? 2 * L.feat_D + 1 : 1));
    s.chi = o; o += al16<double>((size_t)L.nsp * L.nk);
    s.total = o;
    return s;
}

// Deterministic in-order compaction by one warp: writes the indices i < n
// with flag(i) into out, returns the count.
template <typename F>
__device__ __forceinline__ int warp_compact(int n, F flag, int *out) {
    int lane = threadIdx.x & 31, cnt = 0;
    for (int i0 = 0; i0 < n; i0 += 32) {
        int i = i0 + lane;
        bool f = i < n && flag(i);
        unsigned m = __ballot_sync(0xffffffffu, f);
        if (f) out[cnt + __popc(m & ((1u << lane) - 1))] = i;
        cnt += __popc(m);
    }
    return cnt;
}

// The same compaction of the non-zero entries of cnt[0..n) as (index, count).
__device__ __forceinline__ int warp_compact_pairs(int n, const int *cnt, int2 *out) {
    int lane = threadIdx.x & 31, tot = 0;
    for (int i0 = 0; i0 < n; i0 += 32) {
        int i = i0 + lane;
        int v = i < n ? cnt[i] : 0;
        unsigned m = __ballot_sync(0xffffffffu, v != 0);
        if (v != 0) out[tot + __popc(m & ((1u << lane) - 1))] = make_int2(i, v);
        tot += __popc(m);
    }
    return tot;
}

// Library entry of a path record {abs | class entry offset << 20, s0, s1, s2}
// under the species accessor sp (mslibrary.py:433-434).
template <typename SpeciesOf>
__device__ __forceinline__ int ms_entry(SpeciesOf sp, int4 rc, int nsp, int nblk) {
    int e = sp(rc.x & 0xFFFFF) * nblk + (rc.x >> 20);
    int pw = 1;
    if (rc.y >= 0) e += sp(rc.y) * pw;
    pw *= nsp;
    if (rc.z >= 0) e += sp(rc.z) * pw;
    pw *= nsp;
    if (rc.w >= 0) e += sp(rc.w) * pw;
    return e;
}

// d = a * b + c on both halves of a pair (one packed FP32x2 FMA, round to
// nearest per half, as two fmaf)
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

template <int PREC>
struct Real {
    typedef float T;
    typedef float2 T2;
};
template <>
struct Real<CHX_FP64> {
    typedef double T;
    typedef double2 T2;
};

// e^{-2 pi i j / nfft} for an integer j reduced mod nfft (nfft a power of 2,
// so 2 j / nfft is exact): sincospi evaluates it to FP32/FP64 rounding.
__device__ __forceinline__ float2 twiddle(int j, float inv_half) {
    float s, c;
    sincospif((float)j * inv_half, &s, &c);
    return make_float2(c, -s);
}
__device__ __forceinline__ double2 twiddle(int j, double inv_half) {
    double s, c;
    sincospi((double)j * inv_half, &s, &c);
    return make_double2(c, -s);
}

// Resample x window x k^w the normalised trial chi s_tr (nsp, nk) into s_u
// [tap][channel] and transform it on the window bins into s_x (channel-major).
// Kept out of line so that its tap loop has the register file to itself: the
// caller keeps many values live across the call.
template <int NSP, int PREC>
__device__ __noinline__ void ft_window(const chx_ladder_t &L, const double *s_tr,
                                       typename Real<PREC>::T *s_u,
                                       typename Real<PREC>::T2 *s_x, int max_split = kMaxSplit) {
    typedef typename Real<PREC>::T real;
    typedef typename Real<PREC>::T2 real2;
    constexpr int MAXCH = 3 * NSP;
    const int tid = threadIdx.x;
    const int nk = L.nk;
    const int nchan = L.nchan, ncoef = L.ncoef, nwin = L.nwin, nkw = L.nkw;
    const int nchp = nchan + (nchan & 1);      // row stride; the pad channel is zero
    for (int q = tid; q < nchan * ncoef; q += blockDim.x) {
        int ch = q / ncoef, j = q - ch * ncoef, e = ch / nkw;
        int id = L.ft_idx[q];
        double va = s_tr[e * nk + id], vb = s_tr[e * nk + id + 1];
        s_u[j * nchp + ch] = (real)((va + (vb - va) * L.ft_frac[q]) * L.ft_w[q]);
    }
    if (nchan & 1)
        for (int j = tid; j < ncoef; j += blockDim.x) s_u[j * nchp + nchan] = (real)0;
    __syncthreads();
    const int fmask = L.nfft - 1;
    const int n0 = L.ft_n0[0];
    if constexpr (PREC != CHX_FP64 && (MAXCH + 1) / 2 <= 3) {
        // FP32, up to 3 channel pairs: two window bins per thread (qa and
        // qb = qa + nbp), so one shared-memory load of a tap's channel pair
        // feeds both; the taps split into ns runs held by ns adjacent lanes,
        // whose partial sums meet by shuffles, the first lane writing the
        // scaled result. Every lane takes the same number of passes, so the
        // shuffles always see the whole warp.
        constexpr int MAXP = (MAXCH + 1) / 2;
        const int npair = nchp / 2;
        const int nbp = (nwin + 1) >> 1;
        const int ns = nbp * 4 <= (int)blockDim.x ? 4 : (nbp * 2 <= (int)blockDim.x ? 2 : 1);
        const int total = nbp * ns;
        const int jper = (ncoef + ns - 1) / ns;
        const float inv_half = 2.0f / (float)L.nfft;
        const int passes = (total + blockDim.x - 1) / blockDim.x;
        for (int pass = 0; pass < passes; ++pass) {
            const int item = pass * blockDim.x + tid;
            const bool valid = item < total;
            const int bp = valid ? item / ns : 0, part = item - (item / ns) * ns;
            const int qa = bp, qb = bp + nbp;
            const bool hasb = valid && qb < nwin;
            const int ma = L.win_bin[qa] & fmask, mb = L.win_bin[hasb ? qb : qa] & fmask;
            const int j0 = valid ? part * jper : 0, j1 = valid ? min(ncoef, j0 + jper) : 0;
            const float2 ra = twiddle(ma, inv_half), rb = twiddle(mb, inv_half);
            float2 are[MAXP], aim[MAXP], bre[MAXP], bim[MAXP];
#pragma unroll
            for (int p = 0; p < MAXP; ++p)
                are[p] = aim[p] = bre[p] = bim[p] = make_float2(0.f, 0.f);
            for (int jb = j0; jb < j1; jb += kReseed) {
                float2 za = twiddle((int)(((long)(n0 + jb) * ma) & fmask), inv_half);
                float2 zb = twiddle((int)(((long)(n0 + jb) * mb) & fmask), inv_half);
                const int je = min(j1, jb + kReseed);
                for (int j = jb; j < je; ++j) {
                    const float2 *uj = (const float2 *)(s_u + j * nchp);
                    const float2 zax = make_float2(za.x, za.x), zay = make_float2(za.y, za.y);
                    const float2 zbx = make_float2(zb.x, zb.x), zby = make_float2(zb.y, zb.y);
#pragma unroll
                    for (int p = 0; p < MAXP; ++p)
                        if (p < npair) {
                            const float2 u = uj[p];
                            are[p] = ffma2(u, zax, are[p]);
                            aim[p] = ffma2(u, zay, aim[p]);
                            bre[p] = ffma2(u, zbx, bre[p]);
                            bim[p] = ffma2(u, zby, bim[p]);
                        }
                    float t = za.x * ra.x - za.y * ra.y;
                    za.y = fmaf(za.x, ra.y, za.y * ra.x);
                    za.x = t;
                    t = zb.x * rb.x - zb.y * rb.y;
                    zb.y = fmaf(zb.x, rb.y, zb.y * rb.x);
                    zb.x = t;
                }
            }
            for (int o = 1; o < ns; o <<= 1) {
#pragma unroll
                for (int p = 0; p < MAXP; ++p) {
                    are[p].x += __shfl_xor_sync(0xffffffffu, are[p].x, o);
                    are[p].y += __shfl_xor_sync(0xffffffffu, are[p].y, o);
                    aim[p].x += __shfl_xor_sync(0xffffffffu, aim[p].x, o);
                    aim[p].y += __shfl_xor_sync(0xffffffffu, aim[p].y, o);
                    bre[p].x += __shfl_xor_sync(0xffffffffu, bre[p].x, o);
                    bre[p].y += __shfl_xor_sync(0xffffffffu, bre[p].y, o);
                    bim[p].x += __shfl_xor_sync(0xffffffffu, bim[p].x, o);
                    bim[p].y += __shfl_xor_sync(0xffffffffu, bim[p].y, o);
                }
            }
            if (valid && part == 0) {
                const double nrm = L.ft_norm;
#pragma unroll
                for (int p = 0; p < MAXP; ++p) {
                    if (2 * p < nchan) {
                        s_x[(2 * p) * nwin + qa] =
                            real2{(real)(are[p].x * nrm), (real)(aim[p].x * nrm)};
                        if (hasb)
                            s_x[(2 * p) * nwin + qb] =
                                real2{(real)(bre[p].x * nrm), (real)(bim[p].x * nrm)};
                    }
                    if (2 * p + 1 < nchan) {
                        s_x[(2 * p + 1) * nwin + qa] =
                            real2{(real)(are[p].y * nrm), (real)(aim[p].y * nrm)};
                        if (hasb)
                            s_x[(2 * p + 1) * nwin + qb] =
                                real2{(real)(bre[p].y * nrm), (real)(bim[p].y * nrm)};
                    }
                }
            }
        }
        __syncthreads();
        return;
    }
    const int nsplit = max(1, min(max_split, (int)blockDim.x / max(nwin, 1)));
    const int jper = (ncoef + nsplit - 1) / nsplit;
    const int nx = nchan * nwin;
    for (int item = tid; item < nsplit * nwin; item += blockDim.x) {
        int part = item / nwin, q = item - part * nwin;
        int m = L.win_bin[q] & fmask;
        int j0 = part * jper, j1 = min(ncoef, j0 + jper);
        const real inv_half = (real)2.0 / (real)L.nfft;
        const real2 rot = twiddle(m, inv_half);
        if constexpr (PREC != CHX_FP64) {
            // FP32: channel pairs (c, c + 1) of the real and of the imaginary
            // sums, one packed fma.rn.f32x2 each per tap
            constexpr int MAXP = (MAXCH + 1) / 2;
            const int npair = nchp / 2;
            float2 are[MAXP], aim[MAXP];
#pragma unroll
            for (int p = 0; p < MAXP; ++p) are[p] = aim[p] = make_float2(0.f, 0.f);
            for (int jb = j0; jb < j1; jb += kReseed) {
                float2 z = twiddle((int)(((long)(n0 + jb) * m) & fmask), inv_half);
                int je = min(j1, jb + kReseed);
                for (int j = jb; j < je; ++j) {
                    const float2 *uj = (const float2 *)(s_u + j * nchp);
                    const float2 zx = make_float2(z.x, z.x), zy = make_float2(z.y, z.y);
#pragma unroll
                    for (int p = 0; p < MAXP; ++p)
                        if (p < npair) {
                            const float2 u = uj[p];
                            are[p] = ffma2(u, zx, are[p]);
                            aim[p] = ffma2(u, zy, aim[p]);
                        }
                    float zr = z.x * rot.x - z.y * rot.y;
                    z.y = fmaf(z.x, rot.y, z.y * rot.x);
                    z.x = zr;
                }
            }
#pragma unroll
            for (int p = 0; p < MAXP; ++p) {
                if (2 * p < nchan)
                    s_x[part * nx + (2 * p) * nwin + q] = real2{are[p].x, aim[p].x};
                if (2 * p + 1 < nchan)
                    s_x[part * nx + (2 * p + 1) * nwin + q] = real2{are[p].y, aim[p].y};
            }
        } else {
            real ar[MAXCH], ai[MAXCH];
#pragma unroll
            for (int c = 0; c < MAXCH; ++c) ar[c] = ai[c] = 0;
            for (int jb = j0; jb < j1; jb += kReseed) {
                real2 z = twiddle((int)(((long)(n0 + jb) * m) & fmask), inv_half);
                int je = min(j1, jb + kReseed);
                for (int j = jb; j < je; ++j) {
                    const real *uj = s_u + j * nchp;
#pragma unroll
                    for (int c = 0; c < MAXCH; ++c)
                        if (c < nchan) {
                            real u = uj[c];
                            ar[c] = fma(u, z.x, ar[c]);
                            ai[c] = fma(u, z.y, ai[c]);
                        }
                    real zx = z.x * rot.x - z.y * rot.y;
                    z.y = fma(z.x, rot.y, z.y * rot.x);
                    z.x = zx;
                }
            }
#pragma unroll
            for (int c = 0; c < MAXCH; ++c)
                if (c < nchan) s_x[part * nx + c * nwin + q] = real2{ar[c], ai[c]};
        }
    }
    __syncthreads();
    for (int o = tid; o < nx; o += blockDim.x) {
        real2 v = s_x[o];
        for (int p = 1; p < nsplit; ++p) {
            real2 w = s_x[p * nx + o];
            v.x += w.x;
            v.y += w.y;
        }
        s_x[o] = real2{(real)(v.x * L.ft_norm), (real)(v.y * L.ft_norm)};
    }
    __syncthreads();
}

// The profiled chi^2 in two passes (method_a_rmc.py:190-227): per channel
// num = Re<m,t> and den = <m,m> (|m| for a magnitude target), the per-edge
// scale s = sum num / sum den over the edge's channels, then
// sum |s m - t|^2 / sigma^2, all in FP64; m(g) comes from getm(g) (g the
// window point). The second pass sums small residuals, so the result keeps
// FP64's relative precision (a one-pass s^2 A - 2 s B + C cancels). With dx
// (a change of chi(R) inside m), *s_d2 = sum s^2 |dx|^2 / sigma^2.
template <int NSP, typename GetM, typename R2>
__device__ void chi2_profiled(const chx_ladder_t &L, GetM getm, const R2 *dx, double *s_num,
                              double *s_den, double *s_sq, double *s_scale, double *s_c2,
                              double *s_d2) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nchan = L.nchan, nwin = L.nwin, nkw = L.nkw;
    for (int ch = warp; ch < nchan; ch += blockDim.x / 32) {
        double nu = 0.0, dn = 0.0, D = 0.0;
        for (int q = lane; q < nwin; q += 32) {
            const long g = (long)ch * nwin + q;
            const double2 m = getm(g);
            const double tr = L.tm_re[g];
            if (L.cplx) {
                const double ti = L.tm_im[g];
                nu += m.x * tr + m.y * ti;
                dn += m.x * m.x + m.y * m.y;
            } else {
                const double mag = sqrt(m.x * m.x + m.y * m.y);
                nu += mag * tr;
                dn += mag * mag;
            }
            if (dx) {
                const double a = dx[g].x, b = dx[g].y;
                D += (a * a + b * b) * L.w2[g];
            }
        }
        nu = warp_sum(nu);
        dn = warp_sum(dn);
        if (dx) D = warp_sum(D);
        if (lane == 0) {
            s_num[ch] = nu;
            s_den[ch] = dn;
            if (dx) s_sq[36 + ch] = D;
        }
    }
    __syncthreads();
    if (tid < NSP) {
        double sc = 1.0;
        if (L.profile) {
            double nu = 0.0, dn = 0.0;
            for (int q = 0; q < nkw; ++q) {
                nu += s_num[tid * nkw + q];
                dn += s_den[tid * nkw + q];
            }
            sc = nu / fmax(dn, 1e-30);
        }
        s_scale[tid] = sc;
    }
    __syncthreads();
    for (int ch = warp; ch < nchan; ch += blockDim.x / 32) {
        const double sc = s_scale[ch / nkw];
        double acc = 0.0;
        for (int q = lane; q < nwin; q += 32) {
            const long g = (long)ch * nwin + q;
            const double2 m = getm(g);
            const double sg = L.sm[g];
            if (L.cplx) {
                const double dr = (m.x * sc - L.tm_re[g]) / sg;
                const double di = (m.y * sc - L.tm_im[g]) / sg;
                acc += dr * dr + di * di;
            } else {
                const double mag = sqrt(m.x * m.x + m.y * m.y);
                const double dr = (mag * sc - L.tm_re[g]) / sg;
                acc += dr * dr;
            }
        }
        acc = warp_sum(acc);
        if (lane == 0) s_sq[ch] = acc;
    }
    __syncthreads();
    if (tid == 0) {
        double tot = 0.0, d2 = 0.0;
        for (int ch = 0; ch < nchan; ++ch) {
            tot += s_sq[ch];
            if (dx) {
                const double sc = s_scale[ch / nkw];
                d2 += sc * sc * s_sq[36 + ch];
            }
        }
        *s_c2 = tot / L.nfit;
        if (s_d2) *s_d2 = d2;
    }
    __syncthreads();
}

// The same chi^2 in one pass, anchored at the scale s0 of the slot's
// current state: with r0 = s0 m - t, |s m - t|^2 = |r0|^2 + 2 (s - s0)
// Re(m r0*) + (s - s0)^2 |m|^2, so per channel R = sum |r0|^2 / sigma^2,
// Q = sum Re(m r0*) / sigma^2 and P = sum |m|^2 / sigma^2 are summed with
// num and den in one sweep; R carries the size of chi^2 and the other terms
// are small, so nothing cancels. The weights are the stored 1 / sigma^2
// (w2), so no bin divides; against chi2_profiled's (r / sigma)^2 a state's
// own chi^2 differs by rounding only (a few ulps of chi^2). The channel
// terms are combined by one warp (the absorbers' scales, then one lane per
// channel and a warp sum). *s_d2 as in chi2_profiled.
template <int NSP, typename GetM, typename R2>
__device__ void chi2_anchored(const chx_ladder_t &L, GetM getm, const R2 *dx, const double *s0,
                              double *s_num, double *s_den, double *s_sq, double *s_scale,
                              double *s_c2, double *s_d2) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nchan = L.nchan, nwin = L.nwin, nkw = L.nkw;
    const bool cplx = L.cplx;
    for (int ch = warp; ch < nchan; ch += blockDim.x / 32) {
        const double sa = s0[ch / nkw];
        double nu = 0.0, dn = 0.0, R = 0.0, Q = 0.0, Pp = 0.0, D = 0.0;
        for (int q = lane; q < nwin; q += 32) {
            const long g = (long)ch * nwin + q;
            const double2 m = getm(g);
            const double tr = L.tm_re[g], w = L.w2[g];
            const double mm = m.x * m.x + m.y * m.y;
            if (cplx) {
                const double ti = L.tm_im[g];
                nu += m.x * tr + m.y * ti;
                dn += mm;
                const double rr = m.x * sa - tr, ri = m.y * sa - ti;
                R += (rr * rr + ri * ri) * w;
                Q += (m.x * rr + m.y * ri) * w;
            } else {
                const double mag = sqrt(mm);
                nu += mag * tr;
                dn += mm;
                const double rr = mag * sa - tr;
                R += rr * rr * w;
                Q += mag * rr * w;
            }
            Pp += mm * w;
            const double a = dx[g].x, b = dx[g].y;
            D += (a * a + b * b) * w;
        }
        nu = warp_sum(nu);
        dn = warp_sum(dn);
        R = warp_sum(R);
        Q = warp_sum(Q);
        Pp = warp_sum(Pp);
        D = warp_sum(D);
        if (lane == 0) {
            s_num[ch] = nu;
            s_den[ch] = dn;
            s_sq[ch] = R;
            s_sq[12 + ch] = Q;
            s_sq[24 + ch] = Pp;
            s_sq[36 + ch] = D;
        }
    }
    __syncthreads();
    if (warp == 0) {
        double sc_l = 1.0;      // lane e < NSP: absorber e's profiled scale
        if (lane < NSP && L.profile) {
            double nu = 0.0, dn = 0.0;
            for (int q = 0; q < nkw; ++q) {
                nu += s_num[lane * nkw + q];
                dn += s_den[lane * nkw + q];
            }
            sc_l = nu / fmax(dn, 1e-30);
        }
        if (lane < NSP) s_scale[lane] = sc_l;
        const int e = min(lane / nkw, NSP - 1);
        const double sc = __shfl_sync(0xffffffffu, sc_l, e);
        double t = 0.0, d2 = 0.0;
        if (lane < nchan) {     // lane ch: channel ch's terms
            const double ds = sc - s0[e];
            t = s_sq[lane];
            if (ds != 0.0) t += ds * (2.0 * s_sq[12 + lane] + ds * s_sq[24 + lane]);
            d2 = sc * sc * s_sq[36 + lane];
        }
        t = warp_sum(t);
        d2 = warp_sum(d2);
        if (lane == 0) {
            *s_c2 = t / L.nfit;
            if (s_d2) *s_d2 = d2;
        }
    }
    __syncthreads();
}

// The change's window transform on the tensor cores, FP32C with the kept
// chi(R): the normalised change s_tr (nsp, nk) is resampled, windowed and
// weighted by k^w as in ft_window, rounded to BF16 hi + lo (lo = the rest),
// and X = W^T U is formed by mma m16n8k16 with the split-BF16 products
// hi.hi + hi.lo + lo.hi accumulated in FP32 (W^T and its split prepared on
// the host in A-fragment order, ft_frag). U sits in shared memory
// channel-major with a row stride of KP + 8 taps, so the eight rows a B
// fragment reads fall in different banks. Each warp owns m tiles (16 rows:
// re/im of 8 window bins) and all n tiles (8 channels each); s_x receives
// the change's chi(R) (channel-major, as ft_window writes it).
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint4 &a, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
}

template <int NSP>
__device__ __noinline__ void ft_window_tc(const chx_ladder_t &L, const double *s_tr,
                                          uint16_t *s_ub, float2 *s_x) {
    constexpr int MAXNT = (3 * NSP + 7) / 8;        // n tiles of 8 channels
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    const int nk = L.nk, nchan = L.nchan, ncoef = L.ncoef, nkw = L.nkw, nwin = L.nwin;
    const int mtn = L.ft_mt, ktn = L.ft_kt;
    const int KS = ktn * 16 + 8;                    // row stride (taps) of U
    const int nnt = (nchan + 7) >> 3, NP = nnt * 8;
    uint16_t *uh = s_ub, *ul = s_ub + (long)NP * KS;
    // the resample, one tap column per thread across the channel rows: the
    // row's absorber (ch / nkw, nkw <= 3, by multiply and shift) and offsets
    // are uniform over the warp, so no index divides
    for (int j = tid; j < KS; j += blockDim.x) {
        const bool tap = j < ncoef;
#pragma unroll 4
        for (int ch = 0; ch < NP; ++ch) {
            float u = 0.f;
            if (tap && ch < nchan) {
                const int e = nkw == 1 ? ch : (nkw == 2 ? ch >> 1 : (ch * 11) >> 5);
                const long g = (long)ch * ncoef + j;
                const int id = __ldg(&L.ft_idx[g]);
                const double va = s_tr[e * nk + id], vb = s_tr[e * nk + id + 1];
                u = (float)((va + (vb - va) * __ldg(&L.ft_frac[g])) * __ldg(&L.ft_w[g]));
            }
            const __nv_bfloat16 h = __float2bfloat16_rn(u);
            const __nv_bfloat16 l = __float2bfloat16_rn(u - __bfloat162float(h));
            uh[ch * KS + j] = __bfloat16_as_ushort(h);
            ul[ch * KS + j] = __bfloat16_as_ushort(l);
        }
    }
    __syncthreads();
    const int gid = lane >> 2, tig = lane & 3;
    const uint4 *Ah = (const uint4 *)L.ft_frag;
    const uint4 *Al = Ah + (long)mtn * ktn * 32;
    for (int mt = warp; mt < mtn; mt += nwarp) {
        // hi.hi in acc, the two correction products in acc2: two shorter
        // dependent chains of MMAs, added at the end
        float acc[MAXNT][4], acc2[MAXNT][4];
#pragma unroll
        for (int t = 0; t < MAXNT; ++t)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[t][r] = acc2[t][r] = 0.f;
        const uint4 *ah_p = Ah + (long)mt * ktn * 32 + lane;
        const uint4 *al_p = Al + (long)mt * ktn * 32 + lane;
#pragma unroll 4
        for (int kt = 0; kt < ktn; ++kt) {
            const uint4 ah = __ldcg(ah_p + kt * 32), al = __ldcg(al_p + kt * 32);
            const int k0 = kt * 16 + tig * 2;
#pragma unroll
            for (int t = 0; t < MAXNT; ++t) {
                if (t < nnt) {
                    const int rowo = (t * 8 + gid) * KS + k0;
                    const uint32_t bh0 = *(const uint32_t *)&uh[rowo];
                    const uint32_t bh1 = *(const uint32_t *)&uh[rowo + 8];
                    const uint32_t bl0 = *(const uint32_t *)&ul[rowo];
                    const uint32_t bl1 = *(const uint32_t *)&ul[rowo + 8];
                    mma_bf16(acc[t], ah, bh0, bh1);
                    mma_bf16(acc2[t], ah, bl0, bl1);
                    mma_bf16(acc2[t], al, bh0, bh1);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < MAXNT; ++t)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[t][r] += acc2[t][r];
        // D: c0, c1 at row gid, columns tig*2, tig*2+1; c2, c3 at row gid + 8
#pragma unroll
        for (int t = 0; t < MAXNT; ++t) {
            if (t >= nnt) continue;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int row = mt * 16 + gid + 8 * (r >> 1), col = t * 8 + tig * 2 + (r & 1);
                const int q = row >> 1;
                if (q < nwin && col < nchan) {
                    float *o = (float *)&s_x[col * nwin + q];
                    o[row & 1] = acc[t][r];
                }
            }
        }
    }
    __syncthreads();
}

// Steps 4-5 (and the whole of k_eval_chi2): trial chi(R) on the window bins
// (ft_window), then the profiled chi^2 into *s_c2. In FP32C with xr_base
// (the slot's FP64 chi(R) on the window) s_tr holds a move's change alone:
// the trial chi(R) is xr_base plus its transform, and *s_d2 receives
// sum |change|^2 / sigma^2 * s^2 (for the near-tie bound). max_split: the
// FP64 transform's bin splits (1 for the near-tie buffers).
template <int NSP, int PREC>
__device__ void ft_chi2(const chx_ladder_t &L, const double *s_tr, typename Real<PREC>::T *s_u,
                        typename Real<PREC>::T2 *s_x, double *s_num, double *s_den,
                        double *s_sq, double *s_scale, double *s_c2,
                        const double *xr_base = nullptr, double *s_d2 = nullptr,
                        int max_split = kMaxSplit, const double *xs_base = nullptr) {
    typedef typename Real<PREC>::T real;
    typedef typename Real<PREC>::T2 real2;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nchan = L.nchan, nwin = L.nwin, nkw = L.nkw;
    if constexpr (PREC != CHX_FP64) {
        if (xr_base && L.ft_frag)
            ft_window_tc<NSP>(L, s_tr, (uint16_t *)s_u, (float2 *)s_x);
        else
            ft_window<NSP, PREC>(L, s_tr, s_u, s_x, max_split);
    } else {
        ft_window<NSP, PREC>(L, s_tr, s_u, s_x, max_split);
    }

    if constexpr (PREC != CHX_FP64) {
        if (xr_base) {
            // the trial chi(R) = the slot's FP64 chi(R) + the FP32 transform
            // of the change (added in the order the commit adds it)
            auto getm = [&](long g) {
                const real2 d = s_x[g];
                const double2 b = ((const double2 *)xr_base)[g];
                return make_double2((double)d.x + b.x, (double)d.y + b.y);
            };
            chi2_anchored<NSP>(L, getm, s_x, xs_base, s_num, s_den, s_sq, s_scale, s_c2, s_d2);
            return;
        }
        // one pass: per channel num = Re<m,t>, den = <m,m> (the profiled scale)
        // and A = <m,m>/s^2, B = Re<m,t>/s^2, C = <t,t>/s^2, so that
        // sum |s m - t|^2 / s^2 = s^2 A - 2 s B + C (sums in FP64)
        for (int ch = warp; ch < nchan; ch += blockDim.x / 32) {
            double nu = 0.0, dn = 0.0, A = 0.0, B = 0.0, Cc = 0.0;
            for (int q = lane; q < nwin; q += 32) {
                real2 m = s_x[ch * nwin + q];
                long g = (long)ch * nwin + q;
                double tr = L.tm_re[g], ti = L.cplx ? L.tm_im[g] : 0.0;
                double w = L.w2[g];
                double mr = m.x, mi = m.y;
                if (!L.cplx) {
                    mr = sqrt(mr * mr + mi * mi);
                    mi = 0.0;
                }
                double mt = mr * tr + mi * ti, mm = mr * mr + mi * mi;
                nu += mt;
                dn += mm;
                A += mm * w;
                B += mt * w;
            }
            nu = warp_sum(nu);
            dn = warp_sum(dn);
            A = warp_sum(A);
            B = warp_sum(B);
            Cc = L.tnorm[ch];
            if (lane == 0) {
                s_num[ch] = nu;
                s_den[ch] = dn;
                s_sq[ch] = A;
                s_sq[12 + ch] = B;
                s_sq[24 + ch] = Cc;
            }
        }
        __syncthreads();
        if (tid == 0) {
            double tot = 0.0;
            for (int e = 0; e < NSP; ++e) {
                double s = 1.0;
                if (L.profile) {
                    double nu = 0.0, dn = 0.0;
                    for (int q = 0; q < nkw; ++q) {
                        nu += s_num[e * nkw + q];
                        dn += s_den[e * nkw + q];
                    }
                    s = nu / fmax(dn, 1e-30);
                }
                for (int q = 0; q < nkw; ++q) {
                    int ch = e * nkw + q;
                    tot += s * s * s_sq[ch] - 2.0 * s * s_sq[12 + ch] + s_sq[24 + ch];
                }
            }
            *s_c2 = tot / L.nfit;
        }
        __syncthreads();
    } else {
        // profiled chi^2, the reference's two passes (FP64)
        auto getm = [&](long g) {
            const real2 m = s_x[g];
            return make_double2((double)m.x, (double)m.y);
        };
        chi2_profiled<NSP>(L, getm, (const real2 *)nullptr, s_num, s_den, s_sq, s_scale, s_c2,
                           nullptr);
    }
}

// The change of a move again with FP64 terms, for the near-tie re-check: the
// direct records' FP64 term, the FP64 (shell, type) rows of the table counts
// and the FP64 MS rows of the entry changes (lists as the compaction wrote
// them: direct record indices, then (row, count) pairs of the table, then of
// the MS entries in absorber runs s_msb) into s_dchi. Out of line: the step
// keeps its registers for its hot loops.
template <int NSP>
__device__ __noinline__ void tie_delta64(const chx_ladder_t &L, const PairRec *s_dir,
                                         const int *s_list, int ndirmax, int ndn,
                                         const int *s_msb, int ndir, int ndnz, double *s_dchi) {
    const int nk = L.nk, nn = NSP * NSP;
    const int *l_dir = s_list;
    const int2 *l_dn = (const int2 *)(s_list + ndirmax);
    const int2 *l_ms = l_dn + ndn;
    for (int ik = threadIdx.x; ik < nk; ik += blockDim.x) {
        double acc[NSP];
#pragma unroll
        for (int q = 0; q < NSP; ++q) acc[q] = 0.0;
        if (ndir) {
            KConst<NSP> kc;
            load_kconst<NSP>(kc, L.ktab, L.lamtab, L.dtab, L.ftab, L.s02, nk, ik);
            for (int q = 0; q < ndir; ++q) {
                PairRec d = s_dir[l_dir[q]];
                const int neg = d.t >> 16;
                d.t &= 0xFFFF;
                const double v = rec_term<NSP, CHX_FP64>(d, kc);
                add_by_species<NSP>(acc, d.t / NSP, neg ? -v : v);
            }
        }
        if (L.sstab)
            for (int q = 0; q < ndnz; ++q) {
                const int2 jc = l_dn[q];
                add_by_species<NSP>(acc, (jc.x % nn) / NSP,
                                    (double)jc.y * L.sstab[(long)jc.x * nk + ik]);
            }
#pragma unroll
        for (int a_ = 0; a_ < NSP; ++a_) {
            double sa = 0.0;
            for (int q = s_msb[a_]; q < s_msb[a_ + 1]; ++q) {
                const int2 ec = l_ms[q];
                sa = fma((double)ec.y, L.ms_T[(long)ec.x * nk + ik], sa);
            }
            acc[a_] += sa;
        }
#pragma unroll
        for (int q = 0; q < NSP; ++q) s_dchi[q * nk + ik] = acc[q];
    }
    __syncthreads();
}

// The near-tie re-check's arithmetic (out of line, off the hot path): the
// change in FP64 (tie_delta64), its FP64 window transform in the span the
// step reserves for it, and the trial chi^2 from the slot's FP64 chi(R) plus
// that transform (chi2_anchored, as the step's own chi^2) into *s_c2t.
template <int NSP>
__device__ __noinline__ void tie_recheck(const chx_ladder_t &L, const StepSmem &so,
                                         unsigned char *smem, const PairRec *s_dir,
                                         const int *s_list, int ndirmax, int ndn,
                                         const int *s_msb, int ndir, int ndnz, double *s_dchi,
                                         double *s_tr, const double *CNT, const double *XR,
                                         const double *XS, double *s_num, double *s_den,
                                         double *s_sq, double *s_scale, double *s_c2t) {
    const int nk = L.nk;
    tie_delta64<NSP>(L, s_dir, s_list, ndirmax, ndn, s_msb, ndir, ndnz, s_dchi);
    double *u64 = (double *)(smem + so.u);
    double2 *x64 =
        (double2 *)(smem + so.u + al16<double>((size_t)(L.nchan + (L.nchan & 1)) * L.ncoef));
    for (int q = threadIdx.x; q < NSP * nk; q += blockDim.x)
        s_tr[q] = s_dchi[q] / fmax(CNT[q / nk], 1.0);
    __syncthreads();
    ft_window<NSP, CHX_FP64>(L, s_tr, u64, x64, 1);
    auto getm = [&](long g) {
        const double2 d = x64[g];
        return make_double2(d.x + XR[2 * g], d.y + XR[2 * g + 1]);
    };
    chi2_anchored<NSP>(L, getm, x64, XS, s_num, s_den, s_sq, s_scale, s_c2t, nullptr);
}

// Stage 1 of delayed acceptance for a swap of a and b (species differ),
// run by every thread of the step CTA: the surrogate's input (sites lo < hi,
// their neighbourhoods in the feature order, code NSP for lo and hi
// themselves) into s_codes and the orientation sign into *s_sigma; with the
// screen on, the prediction d^ (*s_dhat), the exact prior change, and the
// stage-1 test min(1, exp(-beta nfit d^ - E)) with its own uniform stream.
// Returns 1 when the screen rejects the move (then recorded as rejected).
template <int NSP>
__device__ __noinline__ int da_stage1(const chx_ladder_t &L, const chx_mlp_t &M,
                                      const uint8_t *s_sp, uint8_t *s_codes, float *s_mpart,
                                      float *s_mh, double *s_de, uint64_t step, int rung, int st,
                                      int a, int b, int nsa, int nsb, bool da_on, float lnb,
                                      float *s_sigma, double *s_dhat, double *s_dast,
                                      int *s_skip, int *err) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int natoms = L.natoms, z = L.ncoord, nn = NSP * NSP;
    auto spc = [s_sp](int i) { return (int)(s_sp[i] & 0x7F); };
    {
        const int lo = a < b ? a : b, hi = a < b ? b : a, D = L.feat_D;
        for (int k = tid; k < 2 * D; k += blockDim.x) {
            const int half = k >= D;
            const int site = __ldg(&L.feat_nbr[(long)(half ? hi : lo) * D + (k - half * D)]);
            int code = NSP;
            if ((unsigned)site >= (unsigned)natoms) atomicOr(err, CHX_DEVERR_INDEX);
            else if (site != a && site != b) code = spc(site);
            s_codes[1 + k] = (uint8_t)code;
        }
        if (tid == 0) {
            const int p = spc(lo), q = spc(hi);
            s_codes[0] = (uint8_t)pair_row(p, q, NSP);
            *s_sigma = p < q ? 1.f : -1.f;
        }
        __syncthreads();
    }
    if (!da_on) return 0;
    const float net = mlp_eval_cta(M, s_codes, lnb, L.slot0 + rung, s_mpart, s_mh);
    if (L.etab) {   // exact prior change of the swap, in both stages
        double de1 = 0.0;
        for (int q = tid; q < 4 * z; q += blockDim.x) {
            const int blk = q / z, o = q - blk * z;
            const int site = (blk < 2) ? a : b, pf = site * z + o;
            const int jn = L.jidx[pf];
            if ((unsigned)jn >= (unsigned)natoms) continue;   // flagged by the pair phase
            if (blk >= 2 && jn == a) continue;
            const int i = (blk & 1) ? jn : site, j = (blk & 1) ? site : jn;
            const int si = spc(i), sj = spc(j);
            const int ni_ = (i == a) ? nsa : ((i == b) ? nsb : si);
            const int nj_ = (j == a) ? nsa : ((j == b) ? nsb : sj);
            const int sh = L.shell[pf];
            de1 += L.etab[sh * nn + ni_ * NSP + nj_] - L.etab[sh * nn + si * NSP + sj];
        }
        de1 = warp_sum(de1);
        if (lane == 0) s_de[warp] = de1;
        __syncthreads();
    }
    if (tid == 0) {
        const double beta = L.beta_rung[rung];
        const double dh = (double)*s_sigma * (double)M.out_scale * (double)net;
        double x1 = beta * dh * L.nfit;
        if (L.etab) {
            double d = 0.0;
            for (int w = 0; w < (int)(blockDim.x / 32); ++w) d += s_de[w];
            x1 += L.energy_beta * d;
        }
        const uint64_t h = splitmix64(splitmix64(L.seed ^ kDaSalt) ^
                                      (step * 0x9E3779B97F4A7C15ULL) ^ ((uint64_t)rung << 32));
        const double u1 = u01(splitmix64(h));
        const int pass = (x1 <= 0.0) || (u1 < exp(-fmin(x1, 60.0)));
        *s_dhat = dh;
        *s_skip = !pass;
        s_dast[0] += 1.0;
        if (pass) {
            s_dast[1] += 1.0;
        } else {
            L.acc_rung[rung] = 0;
            if (L.acc_log) L.acc_log[(long)st * L.nrep + rung] = 0;
        }
    }
    __syncthreads();
    return *s_skip;
}

// DA: built with the delayed-acceptance screen and the swap log (a ladder of
// the launch has a surrogate or a log); without it those paths compile away.
// The Metropolis uniform of (step, rung) when no stream of uniforms is given.
__device__ __forceinline__ double metropolis_u(uint64_t seed, uint64_t stepc, int rung) {
    uint64_t h = splitmix64(splitmix64(seed ^ 0xD1B54A32D192ED03ULL) ^
                            (stepc * 0x9E3779B97F4A7C15ULL) ^ ((uint64_t)rung << 32));
    return u01(splitmix64(h));
}

template <int NSP, int PREC, int NT, int MINB, bool DA>
__global__ void __launch_bounds__(NT, MINB) k_step(const chx_ladder_t *__restrict__ Ls,
                                                         const int *__restrict__ slot_ladder,
                                                         int nslots, int nsteps, StepSmem so,
                                                         uint64_t *__restrict__ stepc,
                                                         int *__restrict__ ticket,
                                                         int *__restrict__ err) {
    typedef typename Real<PREC>::T real;
    typedef typename Real<PREC>::T2 real2;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ chx_ladder_t L;
    __shared__ Proposal prop;
    __shared__ uint64_t s_step, s_base;
    __shared__ int s_rung, s_ndir, s_ndn, s_nhist, s_acc;
    __shared__ double s_num[32], s_den[32], s_sq[48], s_scale[8], s_de[NT / 32];
    __shared__ double s_c2;
    __shared__ int s_msb[NSP + 1];
    __shared__ chx_mlp_t s_mlp;
    __shared__ double s_dhat, s_dast[4];
    __shared__ double s_d2, s_xo, s_xd, s_uu, s_c2t;   // near-tie re-check
    __shared__ int s_tie;
    // near-tie bound of the FP32 terms: per warp, the expected squared
    // weighted chi(R) norm of the change's rounding
    __shared__ double s_e2w[NT / 32];
    __shared__ float s_sigma;
    __shared__ int s_daon, s_skip;
    __shared__ long long s_logi;
    // the slot's best state is written once per launch (or when the undo log
    // fills): the current state with the moves made after the best undone
    __shared__ double s_bc2;                 // best chi^2 so far
    __shared__ int s_bimp, s_nu, s_flush;    // best improved, undo entries, flush now
    __shared__ int s_gst, s_dsp, s_posd;     // best_pos stale, displaced since, copy pos
    __shared__ int u_a[kUndo], u_b[kUndo];
    __shared__ uint8_t u_sa[kUndo], u_sb[kUndo], u_sw[kUndo];
    __shared__ double u_p[kUndo][3];
    __shared__ int s_wcnt[NT / 32];          // non-zero MS entries per warp segment
    // the next step's proposal draws and Metropolis uniform, drawn ahead by
    // the last thread while the others work on the current step (they do
    // not depend on the state); double-buffered by step parity
    __shared__ ProposalDraws s_drw[2];
    __shared__ double s_umet[2];
    // the slot's current chi^2 and its rung's inverse temperature (only this
    // CTA writes the one, the other is fixed for the launch)
    __shared__ double s_c2cur, s_beta;
    // the slot's anchored scales (its FP64 chi(R)'s profiled scale per
    // absorber), kept here beside their global copy
    __shared__ double s_xs[NSP];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int slot = blockIdx.x;
    {
        const int *src = (const int *)&Ls[slot_ladder[slot]];
        int *dst = (int *)&L;
        for (int q = tid; q < (int)(sizeof(chx_ladder_t) / 4); q += blockDim.x) dst[q] = src[q];
    }
    __syncthreads();
    const int c = slot - L.slot0;
    const int natoms = L.natoms, z = L.ncoord, nk = L.nk, nn = NSP * NSP;
    const int maxaff = 4 * z;
    const int nent = L.ms_nblk ? NSP * L.ms_nblk : 0;
    const int ndn = L.nshell * nn;
    int *Sg = L.species + (long)c * natoms;
    double *P = L.pos + (long)c * natoms * 3;
    uint8_t *MVg = L.moved + (long)c * natoms;

    real *s_u = (real *)(smem + so.u);
    real2 *s_x = (real2 *)(smem + so.x);
    double *s_tr = (double *)(smem + so.tr);
    double *s_dchi = (double *)(smem + so.dchi);
    PairRec *s_dir = (PairRec *)(smem + so.dir);
    int *s_dirv = (int *)(smem + so.dirv);
    int *s_hist = (int *)(smem + so.hist);
    int *s_dn = (int *)(smem + so.dn);
    int *s_list = (int *)(smem + so.list);
    uint8_t *s_sp = (uint8_t *)(smem + so.sp);
    uint16_t *s_nb = (uint16_t *)(smem + so.nb);
    uint32_t *s_nbm = (uint32_t *)(smem + so.nbm);
    double *s_chi = (double *)(smem + so.chi);
    uint8_t *s_codes = (uint8_t *)(smem + so.cd);
    float *s_mpart = (float *)(smem + so.x);       // surrogate scratch, shares the
    float *s_mh = s_mpart + (NT / 32) * 256;       // transform's region
    auto spc = [s_sp](int i) { return (int)(s_sp[i] & 0x7F); };
    // write the best state (every thread calls it, with s_bimp set): species
    // and, if they changed since best_pos was written, positions; then undo
    // the moves logged after the best point, newest first
    auto flush_best = [&]() {
        int *B = L.best_sp + (long)c * natoms;
        double *BP = L.best_pos + (long)c * natoms * 3;
        for (int q = tid; q < natoms; q += blockDim.x) B[q] = s_sp[q] & 0x7F;
        if (s_posd)
            for (int q = tid; q < 3 * natoms; q += blockDim.x) BP[q] = P[q];
        __syncthreads();
        if (tid == 0) {
            int disp_after = 0;
            for (int u = s_nu - 1; u >= 0; --u) {
                B[u_a[u]] = u_sa[u];
                B[u_b[u]] = u_sb[u];
                if (!u_sw[u]) {
                    disp_after = 1;
                    if (s_posd)
                        for (int x = 0; x < 3; ++x) BP[3 * u_a[u] + x] = u_p[u][x];
                }
            }
            L.best_chi2[c] = s_bc2;
            // best_pos now equals pos unless a displacement came after the best
            s_gst = s_posd ? disp_after : (s_gst || s_dsp);
            s_dsp = 0;
            s_bimp = s_nu = s_flush = 0;
        }
        __syncthreads();
    };

    if (tid == 0) {
        s_base = *(volatile uint64_t *)stepc;
        s_rung = L.rung_of[c];
        s_daon = DA && L.mlp != nullptr && L.da_on != nullptr && *L.da_on != 0;
        if (s_daon) s_mlp = *L.mlp;
        for (int q = 0; q < 4; ++q) s_dast[q] = 0.0;
        s_bc2 = L.best_chi2[c];
        s_bimp = s_nu = s_flush = s_dsp = s_posd = 0;
        s_gst = L.best_stale ? L.best_stale[c] : 1;
        s_c2cur = L.chi2[c];
        s_beta = L.beta_rung[s_rung];
        propose_draws(s_drw[0], L.seed, s_base + 1, s_rung, natoms, L.swap_frac);
        s_umet[0] = metropolis_u(L.seed, s_base + 1, s_rung);
    }
    if (tid <= NSP) s_msb[tid] = 0;
    for (int i = tid; i < natoms; i += blockDim.x)
        s_sp[i] = (uint8_t)((Sg[i] & 0x7F) | (MVg[i] ? 0x80 : 0));
    double *CHg = L.chi + (long)c * NSP * nk;
    for (int q = tid; q < NSP * nk; q += blockDim.x) s_chi[q] = CHg[q];
    __syncthreads();
    const bool use_tab = (PREC != CHX_FP64) && L.sstab32 != nullptr;
    const bool use_xr = (PREC != CHX_FP64) && L.xr != nullptr;
    const bool tie_terms = use_xr && L.tie_eps > 0.0 && L.tie_gdiag != nullptr;
    double *XR = use_xr ? L.xr + (long)c * L.nchan * L.nwin * 2 : nullptr;
    double *XS = use_xr ? L.xs + (long)c * NSP : nullptr;
    if (use_xr && !L.xs) {      // the anchored chi^2 needs the state's scales
        if (threadIdx.x == 0) atomicOr(err, CHX_DEVERR_INDEX);
        return;
    }
    if (use_xr && tid < NSP) s_xs[tid] = XS[tid];   // read after the step's first barrier
    const float *msT32 = L.ms_T32;
    const bool da_on = DA && s_daon != 0;
    const bool log_on = DA && L.log_cap > 0 && L.log_codes != nullptr && L.log_y != nullptr;
    const float lnb = logf((float)L.beta_rung[s_rung]);

    for (int st = 0; st < nsteps; ++st) {
        // ---- 1. proposal (one thread)
        if (tid == 0) {
            s_step = s_base + st + 1;
            prop = propose_finish(s_drw[st & 1], spc, P, L.ideal, L.disp_sigma, L.max_disp,
                                  false);
        }
        for (int e = tid; e < nent; e += blockDim.x) s_hist[e] = 0;
        for (int e = tid; e < ndn; e += blockDim.x) s_dn[e] = 0;
        if (tid < NT / 32) s_e2w[tid] = 0.0;
        __syncthreads();
        const int a = prop.a, b = prop.b, nsa = prop.nsa, nsb = prop.nsb, swp = prop.swap;
        if (tid == NT - 1 && st + 1 < nsteps) {
            propose_draws(s_drw[(st + 1) & 1], L.seed, s_step + 1, s_rung, natoms, L.swap_frac);
            s_umet[(st + 1) & 1] = metropolis_u(L.seed, s_step + 1, s_rung);
        }

        // ---- 1b. delayed acceptance, stage 1 (features, prediction, screen)
        const bool feat = swp && (da_on || log_on) && spc(a) != spc(b);
        int skip = 0;
        if (feat)
            skip = da_stage1<NSP>(L, s_mlp, s_sp, s_codes, s_mpart, s_mh, s_de, s_step, s_rung, st,
                                  a, b, nsa, nsb, da_on, lnb, &s_sigma, &s_dhat, s_dast, &s_skip,
                                  err);
        if (skip) {   // rejected by the screen: the state is unchanged
            __syncthreads();
            continue;
        }

        // ---- 2. affected pairs: old/new terms, table counts or direct records.
        // Pair q of block blk is site -> neighbour (even blocks) or
        // neighbour -> site (odd blocks), site = a (blocks 0, 1) or b (2, 3).
        // In FP32C a reverse pair takes its shell, sigma^2 and geometry from the
        // forward pair (the same bond); FP64 reads the reverse pair's own data.
        const int sa_old = spc(a), sb_old = spc(b);
        double de = 0.0;
        for (int q = tid; q < maxaff; q += blockDim.x) {
            int blk = q / z, o = q - blk * z;
            int site = (blk < 2) ? a : b;
            int pf = site * z + o;
            int jn = L.jidx[pf];
            int p = pf;
            if (PREC == CHX_FP64 && (blk & 1)) p = L.rev[pf];
            s_dirv[2 * q] = 0;
            s_dirv[2 * q + 1] = 0;
            if ((unsigned)jn >= (unsigned)natoms || (unsigned)p >= (unsigned)L.npairs) {
                atomicOr(err, CHX_DEVERR_INDEX);
                continue;
            }
            if (blk >= 2 && (b == a || jn == a)) continue;
            const int i = (blk & 1) ? jn : site, j = (blk & 1) ? site : jn;
            int si = spc(i), sj = spc(j);
            int t_old = si * NSP + sj;
            int ni_ = (i == a) ? nsa : ((i == b) ? nsb : si);
            int nj_ = (j == a) ? nsa : ((j == b) ? nsb : sj);
            int t_new = ni_ * NSP + nj_;
            int sh = L.shell[p];
            if (L.etab) de += L.etab[sh * nn + t_new] - L.etab[sh * nn + t_old];
            bool tab_ok = use_tab && L.pair_tab[p] && !(s_sp[i] & 0x80) && !(s_sp[j] & 0x80);
            bool tab_new = tab_ok && swp;  // a displaced atom leaves its site
            if (tab_ok && tab_new) {
                if (t_old != t_new) {
                    atomicSub(&s_dn[sh * nn + t_old], 1);
                    atomicAdd(&s_dn[sh * nn + t_new], 1);
                }
                continue;
            }
            // distance of the pair p = (pi -> pj + shift) before and after the move
            const int pi_ = (PREC == CHX_FP64) ? i : site, pj_ = (PREC == CHX_FP64) ? j : jn;
            const double *sh3 = L.shift + 3 * (long)p;
            const double *pi = P + 3 * (long)pi_, *pj = P + 3 * (long)pj_;
            double dx = pj[0] + sh3[0] - pi[0], dy = pj[1] + sh3[1] - pi[1],
                   dz = pj[2] + sh3[2] - pi[2];
            double r_old = sqrt(dx * dx + dy * dy + dz * dz);
            double r_new = r_old;
            if (!swp) {  // a displacement: atom a moves to prop.np
                const double *ni = (pi_ == a) ? prop.np : pi, *nj = (pj_ == a) ? prop.np : pj;
                dx = nj[0] + sh3[0] - ni[0];
                dy = nj[1] + sh3[1] - ni[1];
                dz = nj[2] + sh3[2] - ni[2];
                r_new = sqrt(dx * dx + dy * dy + dz * dz);
            }
            double s2 = L.sig2[p];
            auto make = [&](double r, int t, int neg) {  // sign kept in bit 16 of t
                PairRec d;
                double reff = r + L.drtab[sh * nn + t];
                d.reff = reff;
                d.s2 = s2 + L.s2tab[sh * nn + t];
                d.c3 = L.c3tab[sh];
                d.inv_r2 = (float)(1.0 / (reff * reff));
                d.t = t | (neg << 16);
                return d;
            };
            if (tab_ok) {
                atomicSub(&s_dn[sh * nn + t_old], 1);
            } else {
                s_dir[2 * q] = make(r_old, t_old, 1);
                s_dirv[2 * q] = 1;
            }
            s_dir[2 * q + 1] = make(r_new, t_new, 0);
            s_dirv[2 * q + 1] = 1;
        }
        if (L.etab) {
            de = warp_sum(de);
            if (lane == 0) s_de[warp] = de;
        }
        // ---- MS entry changes along the paths through a and b: the species of
        // each site's neighbourhood (old | new << 8 | 0x8000 for site a), then
        // two extra slots per site, D: the site itself, D + 1: zero (an unused
        // template position adds nothing), so that the template loop below
        // reads every position the same way, without branches
        const bool do_ms = nent && swp;
        const bool ms_pack = nent < kMsPackMax;
        if (do_ms && ms_pack) {
            // word of neighbourhood slot d of site a (half 0) or b (half 1) at
            // template position pp: (old species | new species << 14) times
            // the position's entry multiplier, plus 1 << 28 for site a; slot
            // D is the site itself, D + 1 an unused position (zero)
            const int D = L.ms_D, nblk = L.ms_nblk;
            for (int it = tid; it < 2 * (D + 2); it += blockDim.x) {
                const int half = it >= D + 2, d = it - half * (D + 2);
                uint32_t so = 0, sn = 0, fa = 0;
                if (d < D) {
                    const int site = __ldg(&L.ms_nbr[(long)(half ? b : a) * D + d]);
                    so = s_sp[site] & 0x7F;
                    sn = site == a ? nsa : (site == b ? nsb : so);
                    fa = site == a;
                } else if (d == D) {
                    so = half ? sb_old : sa_old;
                    sn = half ? nsb : nsa;
                }
                const uint32_t w = so | (sn << 14);
                uint32_t *o = s_nbm + half * 4 * (D + 2) + d;
                o[0] = w * (uint32_t)nblk + (fa << 28);
                o[D + 2] = w + (fa << 28);
                o[2 * (D + 2)] = w * (uint32_t)NSP + (fa << 28);
                o[3 * (D + 2)] = w * (uint32_t)(NSP * NSP) + (fa << 28);
            }
        } else if (do_ms) {
            const int D = L.ms_D;
            for (int d = tid; d < 2 * D; d += blockDim.x) {
                int half = d >= D;
                int site = __ldg(&L.ms_nbr[(long)(half ? b : a) * D + (d - half * D)]);
                int so = s_sp[site] & 0x7F;
                int sn = site == a ? nsa : (site == b ? nsb : so);
                s_nb[d + 2 * half] = (uint16_t)(so | (sn << 8) | (site == a ? 0x8000 : 0));
            }
            if (tid < 4) {
                const int h = tid >> 1, zero = tid & 1;
                s_nb[h * (D + 2) + D + zero] =
                    zero ? (uint16_t)0
                         : (uint16_t)((h ? sb_old : sa_old) | ((h ? nsb : nsa) << 8));
            }
        }
        __syncthreads();
        if (do_ms) {
            const int M = L.ms_M, D = L.ms_D, nblk = L.ms_nblk;
            const uint2 *tpl = (const uint2 *)L.ms_tpl;
            // each template once, resolved at site a (half 0) and site b
            // (half 1): one load feeds two independent lookup chains; a
            // thread loads kTg of its templates before resolving any of them
            constexpr int kTg = 8;
            for (int m0 = tid; m0 < M; m0 += kTg * blockDim.x) {
                uint2 tg[kTg];
#pragma unroll
                for (int r = 0; r < kTg; ++r) {
                    const int m = m0 + r * blockDim.x;
                    tg[r] = m < M ? __ldg(&tpl[m]) : make_uint2(0u, 0u);
                }
#pragma unroll 2
            for (int r = 0; r < kTg; ++r) {
                if (m0 + r * blockDim.x >= M) break;
                const uint2 t = tg[r];
                int eo[2], en[2], hasa[2];
                if (ms_pack) {
                    // one shared load and one add per position (the device
                    // templates index slot D for the site itself, D + 1 for
                    // an unused position)
#pragma unroll
                    for (int half = 0; half < 2; ++half) {
                        const uint32_t *nbm = s_nbm + half * 4 * (D + 2);
                        uint32_t acc = t.x | (t.x << 14);
#pragma unroll
                        for (int pp = 0; pp < 4; ++pp)
                            acc += nbm[pp * (D + 2) + ((t.y >> (8 * pp)) & 0xFF)];
                        eo[half] = (int)(acc & 0x3FFF);
                        en[half] = (int)((acc >> 14) & 0x3FFF);
                        hasa[half] = (int)(acc >> 28);
                    }
                } else {
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    const uint16_t *nb = s_nb + half * (D + 2);
                    eo[half] = en[half] = (int)t.x;
                    hasa[half] = 0;
#pragma unroll
                    for (int pp = 0; pp < 4; ++pp) {
                        const int v = (t.y >> (8 * pp)) & 0xFF;
                        const int mul =
                            pp == 0 ? nblk : (pp == 1 ? 1 : (pp == 2 ? NSP : NSP * NSP));
                        const int w = nb[v < 0xFE ? v : D + (v - 0xFE)];
                        eo[half] += (w & 0x7F) * mul;
                        en[half] += ((w >> 8) & 0x7F) * mul;
                        hasa[half] |= w & 0x8000;
                    }
                }
                }
                // a path through both sites counts once (in the half of site a)
                if (eo[0] != en[0]) {
                    atomicAdd(&s_hist[en[0]], 1);
                    atomicSub(&s_hist[eo[0]], 1);
                }
                if (!hasa[1] && eo[1] != en[1]) {
                    atomicAdd(&s_hist[en[1]], 1);
                    atomicSub(&s_hist[eo[1]], 1);
                }
            }
            }
        }
        __syncthreads();
        // compact, as (index, count) pairs in ascending index order: the MS
        // entries by every warp (each counts the non-zero entries of its
        // segment, then writes them from its offset), then warp 0 the direct
        // records and warp 1 the table counts; the MS list is split into one
        // run per absorber species (entry / nblk)
        int *l_dir = s_list;
        int2 *l_dn = (int2 *)(s_list + 2 * maxaff);
        int2 *l_ms = l_dn + ndn;
        const int nwarp = blockDim.x >> 5;
        const int mseg = (nent && swp) ? ((nent + nwarp - 1) / nwarp + 31) / 32 * 32 : 0;
        const int ms0 = min(nent, warp * mseg), ms1 = min(nent, ms0 + mseg);
        {
            int cw = 0;
            for (int i0 = ms0; i0 < ms1; i0 += 32) {
                const int i = i0 + lane;
                cw += __popc(__ballot_sync(0xffffffffu, i < ms1 && s_hist[i] != 0));
            }
            if (lane == 0) s_wcnt[warp] = cw;
        }
        __syncthreads();
        {
            int off = 0;
            for (int w = 0; w < warp; ++w) off += s_wcnt[w];
            for (int i0 = ms0; i0 < ms1; i0 += 32) {
                const int i = i0 + lane;
                const int v = i < ms1 ? s_hist[i] : 0;
                const unsigned m = __ballot_sync(0xffffffffu, v != 0);
                if (v != 0) l_ms[off + __popc(m & ((1u << lane) - 1))] = make_int2(i, v);
                // list position of each absorber block's first entry, by the
                // warp whose run holds the block's first index
                if (lane < NSP) {
                    const int key = lane * L.ms_nblk, d = key - i0;
                    if (d >= 0 && d < 32 && key < ms1)
                        s_msb[lane] = off + __popc(m & ((1u << d) - 1));
                }
                off += __popc(m);
            }
            if (warp == nwarp - 1) {
                if (lane == 0) s_nhist = off;
                // the end of the last block; with no MS changes, every block empty
                if (lane <= NSP && (lane == NSP || mseg == 0)) s_msb[lane] = off;
            }
        }
        if (warp == 0) {
            int n = warp_compact(2 * maxaff, [&](int i) { return s_dirv[i] != 0; }, l_dir);
            if (lane == 0) s_ndir = n;
        } else if (warp == 1) {
            int n = warp_compact_pairs(ndn, s_dn, l_dn);
            if (lane == 0) s_ndn = n;
        }
        __syncthreads();

        // ---- 3. delta chi(k)
        const int ndir = s_ndir, ndnz = s_ndn, nms = s_nhist;
        const double *CH = s_chi;
        const double *CNT = L.count + (long)c * NSP;
        // what the transform gets at (absorber, k) index o: with the kept
        // FP64 chi(R) the normalised change alone, else the normalised
        // trial chi plus chi_extra (exafs_gpu/forward.py:183-187,
        // chimera/multift.py:60-61)
        auto trial_k = [&](int o, double d, double inv) {
            if (use_xr) return d / inv;
            double v = (CH[o] + d) / inv;
            if (L.chi_extra) v += L.chi_extra[o];
            return v;
        };
        if (PREC != CHX_FP64 && (nent == 0 || msT32 != nullptr)) {
            // FP32 tables: items per (absorber species, k points), each summing
            // only its absorber's direct records, table rows and MS rows.
            // Direct records (pairs with a displaced atom) first, one thread
            // per k over all of them as the per-k sum does, so that their
            // cost spreads evenly whatever absorbers they belong to; their
            // sums seed the per-absorber items below.
            if (ndir) {
                for (int ik = tid; ik < nk; ik += blockDim.x) {
                    double acc[NSP], gab[NSP];
#pragma unroll
                    for (int s = 0; s < NSP; ++s) acc[s] = gab[s] = 0.0;
                    KConst<NSP> kc;
                    load_kconst<NSP>(kc, L.ktab, L.lamtab, L.dtab, L.ftab, L.s02, nk, ik);
                    for (int q = 0; q < ndir; ++q) {
                        PairRec d = s_dir[l_dir[q]];
                        const int neg = d.t >> 16;
                        d.t &= 0xFFFF;
                        const double v = rec_term<NSP, PREC>(d, kc);
                        add_by_species<NSP>(acc, d.t / NSP, neg ? -v : v);
                        if (tie_terms) add_by_species<NSP>(gab, d.t / NSP, v * v);
                    }
#pragma unroll
                    for (int s = 0; s < NSP; ++s) {
                        s_dchi[s * nk + ik] = acc[s];
                        // the records' sum of term^2, read back by the item
                        // of (s, ik) below before it writes the trial there
                        if (tie_terms) s_tr[s * nk + ik] = gab[s];
                    }
                }
                __syncthreads();
            }
            // The FP32 rows are read four k points at a time (the FP32
            // tables' row stride is nk rounded up to a multiple of 4). A lane
            // pair takes one (absorber, k quad) item: lane h sums half of the
            // absorber's MS rows for the whole quad, then the pair trades
            // partial sums, and lane h finishes k points 4 kq + 2 h and
            // 4 kq + 2 h + 1 (the items of one warp share an absorber).
            const int nk4 = (nk + 3) & ~3, npq = nk4 >> 2, npq16 = (npq + 15) & ~15;
            const int h = tid & 1;
            const float2 z2 = make_float2(0.f, 0.f), o2 = make_float2(1.f, 1.f);
            double e2acc = 0.0;
            for (int it = tid >> 1; it < NSP * npq16; it += blockDim.x >> 1) {
                const int sa_ = it / npq16, kq = it - sa_ * npq16;
                // MS rows: the FP32 running sums of this lane's half (k 0-1 in
                // A, k 2-3 in B) and, for the near-tie model, the sums of
                // (count x row)^2 (the rows' FP64 -> FP32 rounding) and of the
                // running sum^2 (the FP32 accumulation's rounding)
                float2 smA = z2, smB = z2, vqA = z2, vqB = z2;
                if (kq < npq) {
                    const int q0 = s_msb[sa_], q1 = s_msb[sa_ + 1], qm = q0 + ((q1 - q0 + 1) >> 1);
                    const int qa = h ? qm : q0, qb = h ? q1 : qm;
                    // eight rows' loads in flight per thread: the phase is bound
                    // by the bytes a CTA keeps in flight from L2
                    if (tie_terms) {
#pragma unroll 8
                        for (int q = qa; q < qb; ++q) {
                            const int2 ec = l_ms[q];
                            const float w = (float)ec.y;
                            const float4 r = __ldcg((const float4 *)&msT32[(long)ec.x * nk4 + 4 * kq]);
                            const float2 pA = ffma2(make_float2(w, w), make_float2(r.x, r.y), z2);
                            const float2 pB = ffma2(make_float2(w, w), make_float2(r.z, r.w), z2);
                            smA = ffma2(pA, o2, smA);
                            smB = ffma2(pB, o2, smB);
                            vqA = ffma2(pA, pA, vqA);
                            vqB = ffma2(pB, pB, vqB);
                            vqA = ffma2(smA, smA, vqA);
                            vqB = ffma2(smB, smB, vqB);
                        }
                    } else {
#pragma unroll 8
                        for (int q = qa; q < qb; ++q) {
                            const int2 ec = l_ms[q];
                            const float w = (float)ec.y;
                            const float4 r = __ldcg((const float4 *)&msT32[(long)ec.x * nk4 + 4 * kq]);
                            smA = ffma2(make_float2(w, w), make_float2(r.x, r.y), smA);
                            smB = ffma2(make_float2(w, w), make_float2(r.z, r.w), smB);
                        }
                    }
                }
                // lane 0 keeps k 0-1 and takes lane 1's half of them, lane 1
                // keeps k 2-3; the halves are added (half 0's rows first), one
                // more FP32 accumulation step
                const float2 sendS = h ? smA : smB, sendV = h ? vqA : vqB;
                float2 rS, rV;
                rS.x = __shfl_xor_sync(0xffffffffu, sendS.x, 1);
                rS.y = __shfl_xor_sync(0xffffffffu, sendS.y, 1);
                rV.x = __shfl_xor_sync(0xffffffffu, sendV.x, 1);
                rV.y = __shfl_xor_sync(0xffffffffu, sendV.y, 1);
                const float2 oS = h ? smB : smA, oV = h ? vqB : vqA;
                const float2 sm = make_float2(oS.x + rS.x, oS.y + rS.y);
                float2 vq = make_float2(oV.x + rV.x, oV.y + rV.y);
                vq = ffma2(sm, sm, vq);
                const int k0 = 4 * kq + 2 * h;
                if (kq >= npq || k0 >= nk) continue;
                const bool k1ok = k0 + 1 < nk;
                double acc0 = 0.0, acc1 = 0.0;
                if (ndir) {
                    acc0 = s_dchi[sa_ * nk + k0];
                    if (k1ok) acc1 = s_dchi[sa_ * nk + k0 + 1];
                }
                if (use_tab) {
                    if (use_xr) {
                        // FP64 (shell, type) rows: few rows, no rounding; four
                        // rows' loads issued before they are summed in order
                        for (int q0 = 0; q0 < ndnz; q0 += 4) {
                            int w4[4];
                            double2 t4[4];
#pragma unroll
                            for (int r = 0; r < 4; ++r) {
                                w4[r] = 0;
                                t4[r] = make_double2(0.0, 0.0);
                                if (q0 + r < ndnz) {
                                    const int2 jc = l_dn[q0 + r];
                                    if ((jc.x % nn) / NSP == sa_) {
                                        const double *t = L.sstab + (long)jc.x * nk + k0;
                                        w4[r] = jc.y;
                                        t4[r].x = __ldg(t);
                                        if (k1ok) t4[r].y = __ldg(t + 1);
                                    }
                                }
                            }
#pragma unroll
                            for (int r = 0; r < 4; ++r) {
                                if (w4[r] == 0) continue;       // another absorber's row
                                acc0 = fma((double)w4[r], t4[r].x, acc0);
                                if (k1ok) acc1 = fma((double)w4[r], t4[r].y, acc1);
                            }
                        }
                    } else {
                        for (int q = 0; q < ndnz; ++q) {
                            const int2 jc = l_dn[q];
                            if ((jc.x % nn) / NSP != sa_) continue;
                            const float2 t =
                                __ldg((const float2 *)&L.sstab32[(long)jc.x * nk4 + k0]);
                            acc0 += (double)((float)jc.y * t.x);
                            acc1 += (double)((float)jc.y * t.y);
                        }
                    }
                }
                acc0 += (double)sm.x;
                acc1 += (double)sm.y;
                const double v0 = (double)vq.x, v1 = (double)vq.y;
                const double inv = fmax(CNT[sa_], 1.0);
                const int o = sa_ * nk + k0;
                if (tie_terms) {
                    // the change's rounding at (sa_, k): variance eps_rec^2 sum
                    // term^2 + eps_tab^2 sum (count x row)^2 + eps_tr^2 change^2
                    // (the transform's rounding, of relative RMS eps_tr = tie_eps,
                    // acts as an independent error on each input), weighted by
                    // the transform's gain at k
                    const double *gd = L.tie_gdiag + (long)sa_ * nk;
                    const double et2 = L.tie_eps * L.tie_eps;
                    const double g0 = ndir ? s_tr[o] : 0.0;
                    e2acc += (kEpsRec * kEpsRec * g0 + kEpsTab * kEpsTab * v0 + et2 * acc0 * acc0) *
                             gd[k0] / (inv * inv);
                    if (k1ok) {
                        const double g1 = ndir ? s_tr[o + 1] : 0.0;
                        e2acc += (kEpsRec * kEpsRec * g1 + kEpsTab * kEpsTab * v1 +
                                  et2 * acc1 * acc1) * gd[k0 + 1] / (inv * inv);
                    }
                }
                s_dchi[o] = acc0;
                s_tr[o] = trial_k(o, acc0, inv);
                if (k1ok) {
                    s_dchi[o + 1] = acc1;
                    s_tr[o + 1] = trial_k(o + 1, acc1, inv);
                }
            }
            if (tie_terms) {
                e2acc = warp_sum(e2acc);
                if (lane == 0) s_e2w[warp] = e2acc;
            }
        } else
        for (int ik = tid; ik < nk; ik += blockDim.x) {
            double acc[NSP];
#pragma unroll
            for (int s = 0; s < NSP; ++s) acc[s] = 0.0;
            if (ndir) {
                KConst<NSP> kc;
                load_kconst<NSP>(kc, L.ktab, L.lamtab, L.dtab, L.ftab, L.s02, nk, ik);
                for (int q = 0; q < ndir; ++q) {
                    PairRec d = s_dir[l_dir[q]];
                    int neg = d.t >> 16;
                    d.t &= 0xFFFF;
                    double v = rec_term<NSP, PREC>(d, kc);
                    add_by_species<NSP>(acc, d.t / NSP, neg ? -v : v);
                }
            }
            if (use_tab) {
#pragma unroll 4
                for (int q = 0; q < ndnz; ++q) {
                    int2 jc = l_dn[q];
                    add_by_species<NSP>(acc, (jc.x % nn) / NSP,
                                        (double)((float)jc.y *
                                                 __ldg(&L.sstab32[(long)jc.x * ((nk + 3) & ~3) + ik])));
                }
            }
            // MS rows, one run per absorber block: independent loads, no divides
#pragma unroll
            for (int a_ = 0; a_ < NSP; ++a_) {
                const int q0 = s_msb[a_], q1 = s_msb[a_ + 1];
                if (PREC == CHX_FP64 || msT32 == nullptr) {
                    double sa = 0.0;
#pragma unroll 8
                    for (int q = q0; q < q1; ++q) {
                        int2 ec = l_ms[q];
                        sa = fma((double)ec.y, __ldg(&L.ms_T[(long)ec.x * nk + ik]), sa);
                    }
                    acc[a_] += sa;
                } else {
                    float sa = 0.f;
#pragma unroll 16
                    for (int q = q0; q < q1; ++q) {
                        int2 ec = l_ms[q];
                        sa = fmaf((float)ec.y, __ldg(&msT32[(long)ec.x * ((nk + 3) & ~3) + ik]), sa);
                    }
                    acc[a_] += (double)sa;
                }
            }
#pragma unroll
            for (int s = 0; s < NSP; ++s) {
                s_dchi[s * nk + ik] = acc[s];
                s_tr[s * nk + ik] = trial_k(s * nk + ik, acc[s], fmax(CNT[s], 1.0));
            }
        }
        __syncthreads();

        // ---- 4-5. trial chi(R) on the window and its profiled chi^2
        ft_chi2<NSP, PREC>(L, s_tr, s_u, s_x, s_num, s_den, s_sq, s_scale, &s_c2, XR, &s_d2,
                           kMaxSplit, s_xs);

        // ---- 6. Metropolis
        if (tid == 0) {
            double c2 = s_c2;
            int rung = s_rung;
            const double beta = s_beta;
            double xo = 0.0;      // the exact terms of x beside the chi^2 change
            if (feat && da_on) {
                // stage 2 of delayed acceptance: the surrogate's error alone
                // (the prior's change cancels between the two stages)
                xo = -beta * s_dhat * L.nfit;
            } else if (L.etab) {
                double d = 0.0;
                for (int w = 0; w < (int)(blockDim.x / 32); ++w) d += s_de[w];
                xo = L.energy_beta * d;
            }
            double x = beta * (c2 - s_c2cur) * L.nfit + xo;
            s_xo = xo;
            if (feat && log_on) {
                const long long li = (long long)(((s_step - 1) * (uint64_t)L.nrep + (uint64_t)c) %
                                                 (uint64_t)L.log_cap);
                L.log_y[4 * li] = s_sigma * (float)(c2 - s_c2cur);
                L.log_y[4 * li + 1] = lnb;
                L.log_y[4 * li + 2] = (float)(L.slot0 + rung);    // chain: ladder and rung
                L.log_y[4 * li + 3] = (float)s_step;
                s_logi = li;
            }
            double u;
            long ui = (long)(s_step - 1);
            if (L.u_stream && ui < L.u_steps) {
                u = L.u_stream[ui * L.nrep + rung];
            } else {
                if (L.u_stream) atomicOr(err, CHX_DEVERR_INDEX);
                u = s_umet[st & 1];
            }
            int acc = (x <= 0.0) || (u < exp(-fmin(x, 60.0)));
            // a near tie: a rounding e(k) of the change (FP32 terms and rows,
            // the transform) moves x by at most beta * 2 (||r|| + ||change||)
            // s ||B e||_W (Cauchy-Schwarz on the chi^2 change; B the window
            // transform, W = 1 / sigma^2), ||B e||_W taken at kTieSigma
            // standard deviations of the rounding model; if x - tau and
            // x + tau decide differently, the test is redone in FP64 below
            s_tie = 0;
            if (tie_terms) {
                const double rn = sqrt(fmax(c2, 0.0) * L.nfit), dn = sqrt(fmax(s_d2, 0.0));
                double e2 = 0.0, smax = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) e2 += s_e2w[w];
                for (int q = 0; q < NSP; ++q) smax = fmax(smax, fabs(s_scale[q]));
                const double tau = beta * 2.0 * (rn + dn) * smax * kTieSigma * sqrt(e2);
                const double xl = x - tau, xh = x + tau;
                const int al = (xl <= 0.0) || (u < exp(-fmin(xl, 60.0)));
                const int ah = (xh <= 0.0) || (u < exp(-fmin(xh, 60.0)));
                if (al != ah) {
                    s_tie = 1;
                    s_uu = u;
                }
            }
            s_acc = acc;
            s_xd = x;
        }
        __syncthreads();
        if (PREC != CHX_FP64 && s_tie) {
            // the R-factor comparison in FP64: the move's change again with
            // FP64 terms (the direct records' FP64 term, the FP64 (shell, type)
            // and MS rows) replacing the FP32 one, its FP64 window transform
            // (in the span of the resampled rows / transform / direct
            // records), and the trial chi^2 from the slot's FP64 chi(R) plus
            // that, against the current chi^2 the same sums gave
            tie_recheck<NSP>(L, so, smem, s_dir, s_list, 2 * maxaff, ndn, s_msb, s_ndir, s_ndn,
                             s_dchi, s_tr, CNT, XR, s_xs, s_num, s_den, s_sq, s_scale, &s_c2t);
            if (tid == 0) {
                const double x = s_beta * (s_c2t - s_c2cur) * L.nfit + s_xo;
                const double u = s_uu;
                const int acc = (x <= 0.0) || (u < exp(-fmin(x, 60.0)));
                if (L.tie_stat) {
                    L.tie_stat[2 * (long)c] += 1.0;
                    if (acc != s_acc) L.tie_stat[2 * (long)c + 1] += 1.0;
                }
                s_acc = acc;
                s_xd = x;
                s_c2 = s_c2t;
            }
            __syncthreads();
        }
        if (tid == 0) {
            const int acc = s_acc, rung = s_rung;
            if (feat && da_on) {
                const double x = s_xd;
                s_dast[3] += x <= 0.0 ? 1.0 : exp(-fmin(x, 60.0));   // stage-2 probability
                if (acc) s_dast[2] += 1.0;
            }
            L.acc_rung[rung] = (uint8_t)acc;
            if (L.acc_log) L.acc_log[(long)st * L.nrep + rung] = (uint8_t)acc;
        }
        __syncthreads();

        if (feat && log_on) {
            const int nsite = 2 * L.feat_D + 1;
            uint8_t *dst = L.log_codes + s_logi * nsite;
            for (int k = tid; k < nsite; k += blockDim.x) dst[k] = s_codes[k];
        }

        // ---- 7. commit
        if (s_acc) {
            for (int q = tid; q < NSP * nk; q += blockDim.x) s_chi[q] += s_dchi[q];
            if (use_xr) {
                const int nx = L.nchan * L.nwin;
                if (tid < NSP) XS[tid] = s_xs[tid] = s_scale[tid];
                if (s_tie) {        // the FP64 transform of the near-tie test's change
                    const double *x64 =
                        (const double *)(smem + so.u +
                                         al16<double>((size_t)(L.nchan + (L.nchan & 1)) * L.ncoef));
                    for (int q = tid; q < 2 * nx; q += blockDim.x) XR[q] += x64[q];
                } else {
                    for (int q = tid; q < nx; q += blockDim.x) {
                        const real2 d = s_x[q];
                        XR[2 * q] += (double)d.x;
                        XR[2 * q + 1] += (double)d.y;
                    }
                }
            }
            if (nent && swp) {
                int *C = L.ms_C + (long)c * nent;
                for (int q = tid; q < nms; q += blockDim.x) C[l_ms[q].x] += l_ms[q].y;
            }
            if (tid == 0) {
                const int n = s_nu;
                const bool logm = s_bimp && !(s_c2 < s_bc2);   // a move after the best point
                if (logm) {
                    u_a[n] = a;
                    u_b[n] = b;
                    u_sa[n] = (uint8_t)sa_old;
                    u_sb[n] = (uint8_t)sb_old;
                    u_sw[n] = (uint8_t)swp;
                }
                s_sp[a] = (uint8_t)((s_sp[a] & 0x80) | nsa);
                s_sp[b] = (uint8_t)((s_sp[b] & 0x80) | nsb);
                Sg[a] = nsa;
                Sg[b] = nsb;
                if (!swp) {
                    if (logm)
                        for (int x = 0; x < 3; ++x) u_p[n][x] = P[3 * a + x];
                    P[3 * a] = prop.np[0];
                    P[3 * a + 1] = prop.np[1];
                    P[3 * a + 2] = prop.np[2];
                    s_sp[a] |= 0x80;
                    MVg[a] = 1;
                    s_dsp = 1;
                }
                L.chi2[c] = s_c2;
                s_c2cur = s_c2;
                L.n_acc[c] += 1;
                if (s_c2 < s_bc2) {          // a new best: the current state
                    s_bc2 = s_c2;
                    s_bimp = 1;
                    s_nu = 0;
                    s_posd = s_gst || s_dsp;
                } else if (logm) {
                    s_nu = n + 1;
                }
                s_flush = s_bimp && s_nu == kUndo;
            }
            __syncthreads();
            if (s_flush) flush_best();
        }
        __syncthreads();
    }  // steps
    for (int q = tid; q < NSP * nk; q += blockDim.x) CHg[q] = s_chi[q];
    __syncthreads();
    if (s_bimp) flush_best();
    if (tid == 0 && L.best_stale) L.best_stale[c] = (uint8_t)(s_gst || s_dsp);
    if (da_on && tid == 0 && L.da_stat)
        for (int q = 0; q < 4; ++q) L.da_stat[(long)c * 4 + q] += s_dast[q];
    __syncthreads();

    // ---- the last CTA of the launch advances the step counter
    if (tid == 0) {
        __threadfence();
        int t = atomicAdd(ticket, 1);
        if (t == nslots - 1) {
            *ticket = 0;
            *(volatile uint64_t *)stepc = s_base + nsteps;
            __threadfence();
        }
    }
}

// chi^2 of each slot's chi (or of chi_in, same layout) without a move: the
// state's initial and end-of-run chi^2 (method_a_rmc.py:180, 437, 448).
template <int NSP, int PREC>
__global__ void __launch_bounds__(kStepThreads) k_eval_chi2(const chx_ladder_t *__restrict__ Ls,
                                                           const int *__restrict__ slot_ladder,
                                                           StepSmem so,
                                                           const double *__restrict__ chi_in,
                                                           const double *__restrict__ count_in,
                                                           double *__restrict__ out,
                                                           const uint8_t *__restrict__ mask) {
    typedef typename Real<PREC>::T real;
    typedef typename Real<PREC>::T2 real2;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ chx_ladder_t L;
    __shared__ double s_num[32], s_den[32], s_sq[48], s_scale[8], s_c2;
    const int tid = threadIdx.x, slot = blockIdx.x;
    if (mask && !mask[slot]) return;
    {
        const int *src = (const int *)&Ls[slot_ladder[slot]];
        int *dst = (int *)&L;
        for (int q = tid; q < (int)(sizeof(chx_ladder_t) / 4); q += blockDim.x) dst[q] = src[q];
    }
    __syncthreads();
    const int c = slot - L.slot0, nk = L.nk;
    real *s_u = (real *)(smem + so.u);
    real2 *s_x = (real2 *)(smem + so.x);
    double *s_tr = (double *)(smem + so.tr);
    const double *CH = chi_in ? chi_in + (long)slot * NSP * nk : L.chi + (long)c * NSP * nk;
    const double *CNT = count_in ? count_in + (long)slot * NSP : L.count + (long)c * NSP;
    for (int q = tid; q < NSP * nk; q += blockDim.x) {
        double v = CH[q] / fmax(CNT[q / nk], 1.0);
        if (L.chi_extra) v += L.chi_extra[q];
        s_tr[q] = v;
    }
    __syncthreads();
    if (PREC != CHX_FP64 && L.xr) {
        // FP32C with the kept chi(R): the transform in FP64 (one bin split,
        // in the span the step reserves for it), and for the slot's own chi
        // its FP64 chi(R) stored for the step
        const int nx = L.nchan * L.nwin;
        double *u64 = (double *)(smem + so.u);
        double2 *x64 =
            (double2 *)(smem + so.u + al16<double>((size_t)(L.nchan + (L.nchan & 1)) * L.ncoef));
        ft_chi2<NSP, CHX_FP64>(L, s_tr, u64, x64, s_num, s_den, s_sq, s_scale, &s_c2, nullptr,
                               nullptr, 1);
        if (!chi_in) {
            double *X = L.xr + (long)c * nx * 2;
            for (int q = tid; q < nx; q += blockDim.x) {
                X[2 * q] = x64[q].x;
                X[2 * q + 1] = x64[q].y;
            }
            if (tid < NSP && L.xs) L.xs[(long)c * NSP + tid] = s_scale[tid];
        }
    } else {
        ft_chi2<NSP, PREC>(L, s_tr, s_u, s_x, s_num, s_den, s_sq, s_scale, &s_c2);
    }
    if (tid == 0) {
        if (out) out[slot] = s_c2;
        else L.chi2[c] = s_c2;      // masked refresh: the slot's own chi^2
    }
}


// ------------------------------------------------------- FP64 re-anchoring
// A fresh FP64 recompute of a slot's chi(k) from its species, positions and
// MS entry counts, in the pair-count form: pairs whose two atoms sit on their
// ideal sites are counted by (shell, pair type) and contracted with the FP64
// (shell, type) term table (the pair sum of the reference's pair-count model,
// chimera/shellmodel.py:411-413, which equals the per-pair sum to rounding),
// displaced pairs take the reference's FP64 term directly (kernels.py:22-29),
// and the MS part is sum_e C_e T_e in FP64 (mslibrary.py:453-457).
//
// The work of one slot is spread over the GPU: k_reanchor_select lists the
// slots to re-anchor (a mask, every slot, or those whose accepted-move
// counter reached a threshold, decided on the device), k_reanchor_part
// computes one (listed slot, chunk of kRaChunk pairs) item per CTA into a
// partial spectrum, and k_reanchor_fin sums a slot's partials in chunk order,
// adds the MS part, writes chi and resets the slot's counter. Late in a run
// displaced atoms make many pairs direct (each an FP64 exp and sin at every
// k), which one CTA per slot would take milliseconds to evaluate.
constexpr int kReanchorChunk = 1024;   // pairs examined per round of a CTA
constexpr int kRaChunk = 1024;         // pairs per work item
constexpr int kRaWindow = 64;          // slots per round of chx_reanchor

struct RaScratch {
    int *due_list, *due_count;
    double *partial;
};

static int ra_nchunks(const chx_ladder_t *H, int nladders) {
    int mx = 0;
    for (int i = 0; i < nladders; ++i) mx = std::max(mx, (H[i].npairs + kRaChunk - 1) / kRaChunk);
    return mx;
}

static size_t ra_partial_stride(const chx_ladder_t *H, int nladders) {
    int nk = 0;
    for (int i = 0; i < nladders; ++i) nk = std::max(nk, H[i].nk);
    return (size_t)H[0].nsp * nk;
}

// partial spectra: per listed slot, its pair chunks then one MS item per
// absorber block
static int64_t ra_bytes(const chx_ladder_t *H, int nladders, int max_due) {
    size_t b = 256 * (size_t)((max_due * sizeof(int) + 255) / 256) + 256;
    b += sizeof(double) * (size_t)max_due * (ra_nchunks(H, nladders) + H[0].nsp) *
         ra_partial_stride(H, nladders);
    return (int64_t)b;
}

static RaScratch ra_carve(void *scratch, int max_due) {
    RaScratch r;
    char *p = (char *)scratch;
    r.due_list = (int *)p;
    p += 256 * ((max_due * sizeof(int) + 255) / 256);
    r.due_count = (int *)p;
    p += 256;
    r.partial = (double *)p;
    return r;
}

// One CTA: the listed slots of [slot_lo, slot_hi) in ascending order, at most
// max_due of them (a due slot beyond the cap waits for the next call). mask
// given: the masked slots; else every > 0: the slots whose counter reached
// it; else all.
__global__ void __launch_bounds__(1024) k_reanchor_select(const chx_ladder_t *__restrict__ Ls,
                                                          const int *__restrict__ slot_ladder,
                                                          int slot_lo, int slot_hi,
                                                          const uint8_t *__restrict__ mask,
                                                          int every, int max_due,
                                                          uint8_t *__restrict__ due, RaScratch R,
                                                          unsigned long long *__restrict__ count) {
    __shared__ int s_warp[32], s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_base = 0;
    __syncthreads();
    for (int s0 = slot_lo; s0 < slot_hi; s0 += blockDim.x) {
        const int slot = s0 + tid;
        bool go = false;
        if (slot < slot_hi) {
            if (mask) {
                go = mask[slot] != 0;
            } else if (every > 0) {
                const chx_ladder_t *L = &Ls[slot_ladder[slot]];
                go = L->n_acc[slot - L->slot0] >= every;
            } else {
                go = true;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, go);
        if (lane == 0) s_warp[warp] = __popc(m);
        __syncthreads();
        int off = s_base;
        for (int w = 0; w < warp; ++w) off += s_warp[w];
        const int pos = off + __popc(m & ((1u << lane) - 1));
        const bool take = go && pos < max_due;
        if (take) R.due_list[pos] = slot;
        if (due && slot < slot_hi) due[slot] = (uint8_t)take;
        __syncthreads();
        if (tid == 0) {
            int tot = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += s_warp[w];
            s_base += tot;
        }
        __syncthreads();
    }
    if (tid == 0) {
        const int n = min(s_base, max_due);
        *R.due_count = n;
        if (count) *count += (unsigned long long)n;
    }
}

// grid (max_due * (nchunks + NSP)): item = (listed slot di, ch), ch < nchunks a
// chunk of kRaChunk pairs, ch = nchunks + a the MS part of absorber block a
template <int NSP>
__global__ void __launch_bounds__(256) k_reanchor_part(const chx_ladder_t *__restrict__ Ls,
                                                       const int *__restrict__ slot_ladder,
                                                       RaScratch R, int nchunks, int stride,
                                                       int *__restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ chx_ladder_t L;
    __shared__ int s_ndir;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int di = blockIdx.x / (nchunks + NSP), ch = blockIdx.x - di * (nchunks + NSP);
    if (di >= *(volatile const int *)R.due_count) return;
    const int slot = R.due_list[di];
    {
        const int *src = (const int *)&Ls[slot_ladder[slot]];
        int *dst = (int *)&L;
        for (int q = tid; q < (int)(sizeof(chx_ladder_t) / 4); q += blockDim.x) dst[q] = src[q];
    }
    __syncthreads();
    const int c = slot - L.slot0;
    const int natoms = L.natoms, z = L.ncoord, nk = L.nk, nn = NSP * NSP;
    if (ch >= nchunks) {
        // the MS part of absorber block a: sum_e C_e T_e over its entries, in
        // entry order, the counts staged in shared memory first
        const int a = ch - nchunks, nblk = L.ms_nblk;
        if (!nblk) return;                 // no MS: fin adds nothing
        int *s_cnt = (int *)smem;
        const int *C = L.ms_C + (long)c * NSP * nblk + (long)a * nblk;
        for (int e = tid; e < nblk; e += blockDim.x) s_cnt[e] = C[e];
        __syncthreads();
        double *out = R.partial + ((long)di * (nchunks + NSP) + ch) * stride;
        const double *T = L.ms_T + (long)a * nblk * nk;
        for (int ik = tid; ik < nk; ik += blockDim.x) {
            double acc = 0.0;
#pragma unroll 8
            for (int e = 0; e < nblk; ++e) {
                const int n = s_cnt[e];
                if (n) acc += (double)n * T[(long)e * nk + ik];
            }
            out[ik] = acc;
        }
        return;
    }
    const int p0 = ch * kRaChunk;
    if (p0 >= L.npairs) return;            // beyond this ladder's pairs: fin skips it
    const int p1 = min(L.npairs, p0 + kRaChunk);
    const int nbins = L.nshell * nn;
    const int nwarps = blockDim.x / 32;
    PairRec *s_rec = (PairRec *)smem;                        // direct pairs of a round
    int *s_hist = (int *)(s_rec + kReanchorChunk);           // (nwarps, nbins)
    int *s_dir = s_hist + nwarps * nbins;                    // their pair offsets
    uint8_t *s_flag = (uint8_t *)(s_dir + kReanchorChunk);   // 1: the pair is direct
    uint8_t *s_sp = s_flag + kReanchorChunk;                 // species | moved << 7
    const int *Sg = L.species + (long)c * natoms;
    const uint8_t *MVg = L.moved + (long)c * natoms;
    const double *P = L.pos + (long)c * natoms * 3;
    for (int q = tid; q < nwarps * nbins; q += blockDim.x) s_hist[q] = 0;
    // the k-point constants of the (up to two) k points of this thread
    KConst<NSP> kc[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int ik = tid + h * blockDim.x;
        if (ik < nk) load_kconst<NSP>(kc[h], L.ktab, L.lamtab, L.dtab, L.ftab, L.s02, nk, ik);
    }
    // the species of the atoms this chunk's pairs touch: all of them (a chunk
    // spans ~kRaChunk / z absorbers, but its neighbours reach anywhere)
    for (int i = tid; i < natoms; i += blockDim.x)
        s_sp[i] = (uint8_t)((Sg[i] & 0x7F) | (MVg[i] ? 0x80 : 0));
    __syncthreads();
    const bool tab = L.sstab != nullptr;
    int *hw = s_hist + warp * nbins;
    // thread tid owns k = tid and tid + blockDim (nk <= 2 * blockDim)
    double acc[2][NSP];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int s = 0; s < NSP; ++s) acc[h][s] = 0.0;
    for (int c0 = p0; c0 < p1; c0 += kReanchorChunk) {
        const int n = min(kReanchorChunk, p1 - c0);
        for (int q = tid; q < n; q += blockDim.x) {
            int p = c0 + q, i = p / z, j = L.jidx[p];
            uint8_t direct = 0;
            if ((unsigned)j >= (unsigned)natoms) {
                atomicOr(err, CHX_DEVERR_INDEX);
            } else {
                int wi = s_sp[i], wj = s_sp[j];
                if (tab && L.pair_tab[p] && !((wi | wj) & 0x80))
                    atomicAdd(&hw[L.shell[p] * nn + (wi & 0x7F) * NSP + (wj & 0x7F)], 1);
                else
                    direct = 1;
            }
            s_flag[q] = direct;
        }
        __syncthreads();
        if (warp == 0) {                       // in-order list of the round's direct pairs
            int cnt = warp_compact(n, [&](int q) { return s_flag[q] != 0; }, s_dir);
            if (lane == 0) s_ndir = cnt;
        }
        __syncthreads();
        const int nd = s_ndir;
        // one record per direct pair, built in parallel (geometry and the
        // per-(shell, type) offsets: everything that does not depend on k)
        for (int q = tid; q < nd; q += blockDim.x) {
            const int p = c0 + s_dir[q];
            const int i = p / z, j = L.jidx[p];
            const double *sh3 = L.shift + 3 * (long)p;
            const double *pi = P + 3 * (long)i, *pj = P + 3 * (long)j;
            const double dx = pj[0] + sh3[0] - pi[0], dy = pj[1] + sh3[1] - pi[1],
                         dz = pj[2] + sh3[2] - pi[2];
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const int t = (s_sp[i] & 0x7F) * NSP + (s_sp[j] & 0x7F), sh = L.shell[p];
            PairRec d;
            d.reff = r + L.drtab[sh * nn + t];
            d.s2 = L.sig2[p] + L.s2tab[sh * nn + t];
            d.c3 = L.c3tab[sh];
            d.inv_r2 = (float)(1.0 / (d.reff * d.reff));
            d.t = t;
            s_rec[q] = d;
        }
        __syncthreads();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int ik = tid + h * blockDim.x;
            if (ik >= nk || nd == 0) continue;
            for (int q = 0; q < nd; ++q) {
                const PairRec d = s_rec[q];
                add_by_species<NSP>(acc[h], d.t / NSP, rec_term<NSP, CHX_FP64>(d, kc[h]));
            }
        }
        __syncthreads();
    }
    for (int bb = tid; bb < nbins; bb += blockDim.x) {
        int v = 0;
        for (int w = 0; w < nwarps; ++w) v += s_hist[w * nbins + bb];
        s_hist[bb] = v;
    }
    __syncthreads();
    double *out = R.partial + ((long)di * (nchunks + NSP) + ch) * stride;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int ik = tid + h * blockDim.x;
        if (ik >= nk) continue;
        if (tab)
            for (int bb = 0; bb < nbins; ++bb) {
                int n = s_hist[bb];
                if (n)
                    add_by_species<NSP>(acc[h], (bb % nn) / NSP,
                                        (double)n * L.sstab[(long)bb * nk + ik]);
            }
#pragma unroll
        for (int s = 0; s < NSP; ++s) out[s * nk + ik] = acc[h][s];
    }
}

// grid (max_due): chi of listed slot di = its partials in chunk order + the
// MS part; the slot's accepted-move counter restarts
template <int NSP>
__global__ void __launch_bounds__(256) k_reanchor_fin(const chx_ladder_t *__restrict__ Ls,
                                                      const int *__restrict__ slot_ladder,
                                                      RaScratch R, int nchunks, int stride) {
    const int di = blockIdx.x;
    if (di >= *(volatile const int *)R.due_count) return;
    const int slot = R.due_list[di];
    __shared__ chx_ladder_t L;
    {
        const int *src = (const int *)&Ls[slot_ladder[slot]];
        int *dst = (int *)&L;
        for (int q = threadIdx.x; q < (int)(sizeof(chx_ladder_t) / 4); q += blockDim.x)
            dst[q] = src[q];
    }
    __syncthreads();
    const int c = slot - L.slot0, nk = L.nk;
    const int nch = (L.npairs + kRaChunk - 1) / kRaChunk;
    double *CHg = L.chi + (long)c * NSP * nk;
    const double *part = R.partial + (long)di * (nchunks + NSP) * stride;
    for (int ik = threadIdx.x; ik < nk; ik += blockDim.x) {
        double acc[NSP];
#pragma unroll
        for (int s = 0; s < NSP; ++s) acc[s] = 0.0;
#pragma unroll 8
        for (int q = 0; q < nch; ++q)
#pragma unroll
            for (int s = 0; s < NSP; ++s) acc[s] += part[(long)q * stride + s * nk + ik];
        if (L.ms_nblk)                     // the MS items, one per absorber block
#pragma unroll
            for (int a = 0; a < NSP; ++a) acc[a] += part[(long)(nchunks + a) * stride + ik];
#pragma unroll
        for (int s = 0; s < NSP; ++s) CHg[s * nk + ik] = acc[s];
    }
    if (threadIdx.x == 0) L.n_acc[c] = 0;
}

// ------------------------------------------------------- replica exchange
// One thread per ladder (method_a_rmc.py:332-373 with the uniforms from a
// counter stream): rung pairs (i, i+1) from a random parity, d >= 0 or
// u < exp(max(d, -60)); an accepted pair swaps which slots the two rungs hold.
constexpr int kMaxExchRungs = 1024;

// One CTA per ladder: the rungs' slots and the pairs' d are gathered in
// parallel, one thread walks the pairs in order drawing a uniform only where
// d < 0 (the order of the stream), and the accepted pairs are applied in
// parallel (pairs of one parity touch disjoint rungs and slots).
__global__ void __launch_bounds__(128) k_exchange(const chx_ladder_t *__restrict__ Ls,
                                                  int nladders,
                                                  const uint64_t *__restrict__ round_key) {
    __shared__ int s_slot[kMaxExchRungs];
    __shared__ double s_d[kMaxExchRungs];
    __shared__ uint8_t s_ok[kMaxExchRungs];
    __shared__ int s_start;
    const int li = blockIdx.x, tid = threadIdx.x;
    if (li >= nladders) return;
    const chx_ladder_t &L = Ls[li];
    const int n = min(L.nrep, kMaxExchRungs);
    for (int i = tid; i < n; i += blockDim.x) s_slot[i] = L.slot_of[i];
    __syncthreads();
    for (int i = tid; i < n - 1; i += blockDim.x)
        s_d[i] = (L.beta_rung[i] - L.beta_rung[i + 1]) * (L.chi2[s_slot[i]] - L.chi2[s_slot[i + 1]]) *
                 L.nfit;
    __syncthreads();
    if (tid == 0) {
        const uint64_t round = *(volatile const uint64_t *)round_key;
        uint64_t h = splitmix64(splitmix64(L.seed ^ 0x5851F42D4C957F2DULL) ^
                                (round * 0x9E3779B97F4A7C15ULL));
        h = splitmix64(h);
        const int start = (u01(h) < 0.5) ? 0 : 1;
        s_start = start;
        for (int i = start; i < n - 1; i += 2) {
            const double d = s_d[i];
            bool ok = d >= 0.0;
            if (!ok) {
                h = splitmix64(h);
                ok = u01(h) < exp(fmax(d, -60.0));
            }
            s_ok[i] = (uint8_t)ok;
        }
    }
    __syncthreads();
    for (int i = s_start + 2 * tid; i < n - 1; i += 2 * blockDim.x) {
        L.exch_att[i] += 1;
        if (s_ok[i]) {
            const int si = s_slot[i], sj = s_slot[i + 1];
            L.exch_acc[i] += 1;
            L.slot_of[i] = sj;
            L.slot_of[i + 1] = si;
            L.rung_of[sj] = i;
            L.rung_of[si] = i + 1;
        }
    }
}

// A host-decided permutation: rung i takes the state rung order[i] held.
__global__ void k_apply_exchange(const chx_ladder_t *__restrict__ Ls, int ladder,
                                 const int *__restrict__ order) {
    const chx_ladder_t &L = Ls[ladder];
    if (threadIdx.x != 0) return;
    int tmp[1024];
    int n = min(L.nrep, 1024);
    for (int i = 0; i < n; ++i) {
        int o = order[i];
        tmp[i] = ((unsigned)o < (unsigned)n) ? L.slot_of[o] : L.slot_of[i];
    }
    for (int i = 0; i < n; ++i) {
        L.slot_of[i] = tmp[i];
        L.rung_of[tmp[i]] = i;
    }
}

// sstab[(sh*nn + t)][k] = the term of an ideal pair of shell sh and type t
template <int NSP>
__global__ void k_shell_table(chx_ladder_t L, const double *__restrict__ rshell,
                              const double *__restrict__ s2shell, double *__restrict__ sstab) {
    int jt = blockIdx.x, nn = NSP * NSP;
    int sh = jt / nn, t = jt % nn;
    for (int ik = threadIdx.x; ik < L.nk; ik += blockDim.x) {
        KPoint kp{L.ktab[ik], L.lamtab[ik]};
        sstab[(long)jt * L.nk + ik] = term64(rshell[sh], t, sh, s2shell[sh], ik, L.nk, NSP, kp,
                                             L.ftab, L.dtab, L.drtab, L.c3tab, L.s2tab, L.s02);
    }
}

template <int NSP, int PREC, int NT, int MINB, bool DA>
static int launch_step_nt(const chx_ladder_t *d_ladders, const int *slot_ladder, int nslots,
                          int nsteps, const StepSmem &so, size_t smem, uint64_t *d_stepc,
                          int *d_ticket, int *d_err, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(k_step<NSP, PREC, NT, MINB, DA>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "sampler_step attribute");
    k_step<NSP, PREC, NT, MINB, DA><<<nslots, NT, smem, st>>>(d_ladders, slot_ladder, nslots,
                                                              nsteps, so, d_stepc, d_ticket,
                                                              d_err);
    CHX_CHECK_LAUNCH("sampler_step");
    return CHX_OK;
}

template <int NSP, int PREC, bool DA>
static int launch_step_da(const chx_ladder_t *d_ladders, const int *slot_ladder, int nslots,
                          int nsteps, int threads, int min_blocks, const StepSmem &so,
                          size_t smem, uint64_t *d_stepc, int *d_ticket, int *d_err,
                          cudaStream_t st) {
    if (threads == 128)
        return launch_step_nt<NSP, PREC, 128, 6, DA>(d_ladders, slot_ladder, nslots, nsteps, so,
                                                     smem, d_stepc, d_ticket, d_err, st);
    if (min_blocks == 4)
        return launch_step_nt<NSP, PREC, 256, 4, DA>(d_ladders, slot_ladder, nslots, nsteps, so,
                                                     smem, d_stepc, d_ticket, d_err, st);
    return launch_step_nt<NSP, PREC, 256, 3, DA>(d_ladders, slot_ladder, nslots, nsteps, so,
                                                 smem, d_stepc, d_ticket, d_err, st);
}

template <int NSP, int PREC>
static int launch_step(const chx_ladder_t *d_ladders, const int *slot_ladder, int nslots,
                       int nsteps, int threads, int min_blocks, const StepSmem &so, size_t smem,
                       uint64_t *d_stepc, int *d_ticket, int *d_err, bool da, cudaStream_t st) {
    if (da)
        return launch_step_da<NSP, PREC, true>(d_ladders, slot_ladder, nslots, nsteps, threads,
                                               min_blocks, so, smem, d_stepc, d_ticket, d_err,
                                               st);
    return launch_step_da<NSP, PREC, false>(d_ladders, slot_ladder, nslots, nsteps, threads,
                                            min_blocks, so, smem, d_stepc, d_ticket, d_err, st);
}

template <int NSP, int PREC>
static int launch_eval(const chx_ladder_t *d_ladders, const int *slot_ladder, int nslots,
                       const StepSmem &so, size_t smem, const double *chi_in,
                       const double *count_in, double *out, const uint8_t *mask,
                       cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(k_eval_chi2<NSP, PREC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "eval_chi2 attribute");
    k_eval_chi2<NSP, PREC><<<nslots, kStepThreads, smem, st>>>(d_ladders, slot_ladder, so,
                                                               chi_in, count_in, out, mask);
    CHX_CHECK_LAUNCH("eval_chi2");
    return CHX_OK;
}

// One carve-up for all ladders of a launch: the largest extent of each field.
static int plan_ladders(const chx_ladder_t *H, int nladders, int precision, StepSmem *out,
                        size_t *bytes) {
    int nsp = H[0].nsp;
    StepSmem mx{};
    for (int i = 0; i < nladders; ++i) {
        const chx_ladder_t &L = H[i];
        CHX_REQUIRE(L.nsp == nsp, "sampler: one launch needs one species count");
        CHX_REQUIRE(!L.ms_nblk || (L.ms_tpl && L.ms_nbr && L.ms_D > 0 && L.ms_D < 0xFD &&
                                   L.ms_M > 0 && L.natoms < 65536),
                    "sampler: ladder %d has incomplete multiple-scattering templates", i);
        CHX_REQUIRE(L.ncoord > 0 && L.ncoord <= kMaxCoord && L.nk > 0 && L.nkw >= 1 &&
                        L.nkw <= 3 && L.nchan == L.nsp * L.nkw && (L.nfft & (L.nfft - 1)) == 0 &&
                        L.natoms < (1 << 20) && L.nwin > 0,
                    "sampler: ladder %d outside the built limits", i);
        CHX_REQUIRE(!L.ft_frag || (L.xr && L.ft_mt * 16 >= 2 * L.nwin && L.ft_kt * 16 >= L.ncoef &&
                                   L.ft_mt > 0 && L.ft_kt > 0),
                    "sampler: ladder %d has transform fragments that do not cover its window", i);
        CHX_REQUIRE(L.nrep >= 1 && L.nrep <= kMaxExchRungs,
                    "sampler: ladder %d has %d rungs (1..%d)", i, L.nrep, kMaxExchRungs);
        CHX_REQUIRE(!L.mlp || (L.da_on && L.da_stat),
                    "sampler: ladder %d has a surrogate but no da_on word or da_stat", i);
        CHX_REQUIRE(!(L.mlp || L.log_cap > 0) ||
                        (L.feat_nbr && L.feat_D > 0 && L.feat_D <= 127 &&
                         (L.log_cap == 0 || (L.log_codes && L.log_y && L.log_cap > 0))),
                    "sampler: ladder %d has an incomplete surrogate feature set or swap log", i);
        StepSmem s = step_smem(L, precision);
        // field sizes of this ladder, then the running maximum of each
        size_t f[13] = {s.x - s.u, s.dir - s.x, s.dirv - s.dir, s.tr - s.dirv, s.dchi - s.tr,
                        s.hist - s.dchi, s.dn - s.hist, s.list - s.dn, s.sp - s.list,
                        s.nb - s.sp, s.cd - s.nb, s.chi - s.cd, s.total - s.chi};
        size_t *g[13] = {&mx.u, &mx.x, &mx.dir, &mx.dirv, &mx.tr, &mx.dchi, &mx.hist, &mx.dn,
                         &mx.list, &mx.sp, &mx.nb, &mx.cd, &mx.chi};
        for (int q = 0; q < 13; ++q) *g[q] = std::max(*g[q], f[q]);
        mx.tie = std::max(mx.tie, s.tie);
    }
    // the near-tie span u .. dirv must hold the largest FP64 buffers
    {
        const size_t span = mx.u + mx.x + mx.dir + mx.dirv;
        if (span < mx.tie) mx.dirv += (mx.tie - span + 15) / 16 * 16;
    }
    // mx holds field sizes; turn them into offsets
    StepSmem o;
    size_t at = 0;
    o.tie = mx.tie;
    o.u = at; at += mx.u;
    o.x = at; at += mx.x;
    o.dir = at; at += mx.dir;
    o.dirv = at; at += mx.dirv;
    o.tr = at; at += mx.tr;
    o.dchi = at; at += mx.dchi;
    o.hist = at; at += mx.hist;
    o.dn = at; at += mx.dn;
    o.list = at; at += mx.list;
    o.sp = at; at += mx.sp;
    o.nb = at; at += mx.nb;
    o.cd = at; at += mx.cd;
    o.chi = at; at += mx.chi;
    o.total = at;
    CHX_REQUIRE(at <= 220 * 1024, "sampler: %zu bytes of shared memory needed", at);
    *out = o;
    *bytes = at;
    return CHX_OK;
}

}  // namespace chx

using namespace chx;

extern "C" {

int chx_sampler_smem_bytes(const chx_ladder_t *host_ladders, int nladders, int precision) {
    if (!host_ladders || nladders <= 0) return CHX_ERR_ARG;
    StepSmem so;
    size_t bytes = 0;
    int rc = plan_ladders(host_ladders, nladders, precision, &so, &bytes);
    return rc == CHX_OK ? (int)bytes : rc;
}

int chx_shell_table(const chx_ladder_t *L, const double *rshell, const double *s2shell,
                    double *sstab, void *stream) {
    CHX_REQUIRE(L && rshell && s2shell && sstab, "shell_table: bad arguments");
    int n = L->nshell * L->nsp * L->nsp;
    cudaStream_t st = as_stream(stream);
    switch (L->nsp) {
        case 2: k_shell_table<2><<<n, 256, 0, st>>>(*L, rshell, s2shell, sstab); break;
        case 3: k_shell_table<3><<<n, 256, 0, st>>>(*L, rshell, s2shell, sstab); break;
        case 4: k_shell_table<4><<<n, 256, 0, st>>>(*L, rshell, s2shell, sstab); break;
        default: set_error("shell_table: nsp %d not built", L->nsp); return CHX_ERR_UNSUPPORTED;
    }
    CHX_CHECK_LAUNCH("shell_table");
    return CHX_OK;
}

int chx_sampler_step(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders,
                     int nladders, const int *slot_ladder, int nslots, int precision, int nsteps,
                     int threads, int min_blocks, uint64_t *d_stepc, int *d_ticket, int *d_err,
                     void *stream) {
    CHX_REQUIRE(d_ladders && host_ladders && slot_ladder && d_stepc && d_ticket && d_err &&
                    nladders > 0 && nslots > 0 && nsteps > 0,
                "sampler_step: bad arguments");
    CHX_REQUIRE(precision == CHX_FP64 || precision == CHX_FP32C, "sampler_step: bad precision");
    CHX_REQUIRE((threads == 0 && min_blocks == 0) || (threads == 128 && min_blocks == 6) ||
                    (threads == 256 && (min_blocks == 3 || min_blocks == 4)),
                "sampler_step: launch shape (%d, %d) not built; (128, 6), (256, 3) or (256, 4)",
                threads, min_blocks);
    StepSmem so;
    size_t smem = 0;
    int rc = plan_ladders(host_ladders, nladders, precision, &so, &smem);
    if (rc != CHX_OK) return rc;
    cudaStream_t st = as_stream(stream);
    int nsp = host_ladders[0].nsp;
    bool da = false;
    for (int i = 0; i < nladders; ++i)
        da = da || host_ladders[i].mlp != nullptr || host_ladders[i].log_cap > 0;
#define CHX_STEP(N, PR) \
    launch_step<N, PR>(d_ladders, slot_ladder, nslots, nsteps, threads, min_blocks, so, smem, \
                       d_stepc, d_ticket, d_err, da, st)
    if (precision == CHX_FP64) {
        switch (nsp) {
            case 2: return CHX_STEP(2, CHX_FP64);
            case 3: return CHX_STEP(3, CHX_FP64);
            case 4: return CHX_STEP(4, CHX_FP64);
        }
    } else {
        switch (nsp) {
            case 2: return CHX_STEP(2, CHX_FP32C);
            case 3: return CHX_STEP(3, CHX_FP32C);
            case 4: return CHX_STEP(4, CHX_FP32C);
        }
    }
#undef CHX_STEP
    set_error("sampler_step: nsp %d not built", nsp);
    return CHX_ERR_UNSUPPORTED;
}

int chx_eval_chi2(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders, int nladders,
                  const int *slot_ladder, int nslots, int precision, const double *chi_in,
                  const double *count_in, double *out, void *stream) {
    CHX_REQUIRE(d_ladders && host_ladders && slot_ladder && out && nladders > 0 && nslots > 0,
                "eval_chi2: bad arguments");
    StepSmem so;
    size_t smem = 0;
    int rc = plan_ladders(host_ladders, nladders, precision, &so, &smem);
    if (rc != CHX_OK) return rc;
    cudaStream_t st = as_stream(stream);
    int nsp = host_ladders[0].nsp;
#define CHX_EV(N, PR) launch_eval<N, PR>(d_ladders, slot_ladder, nslots, so, smem, chi_in, count_in, out, nullptr, st)
    if (precision == CHX_FP64) {
        switch (nsp) {
            case 2: return CHX_EV(2, CHX_FP64);
            case 3: return CHX_EV(3, CHX_FP64);
            case 4: return CHX_EV(4, CHX_FP64);
        }
    } else {
        switch (nsp) {
            case 2: return CHX_EV(2, CHX_FP32C);
            case 3: return CHX_EV(3, CHX_FP32C);
            case 4: return CHX_EV(4, CHX_FP32C);
        }
    }
#undef CHX_EV
    set_error("eval_chi2: nsp %d not built", nsp);
    return CHX_ERR_UNSUPPORTED;
}

static int reanchor_launch(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders,
                           int nladders, const int *slot_ladder, int nslots, const uint8_t *mask,
                           int every, int max_due, uint8_t *due, unsigned long long *count,
                           void *scratch, int64_t scratch_bytes, int *d_err, cudaStream_t st) {
    int nsp = host_ladders[0].nsp;
    size_t smem = 0;
    for (int i = 0; i < nladders; ++i) {
        const chx_ladder_t &L = host_ladders[i];
        CHX_REQUIRE(L.nsp == nsp, "reanchor: one launch needs one species count");
        CHX_REQUIRE(L.nk <= 512, "reanchor: nk %d above 512", L.nk);
        size_t b = sizeof(PairRec) * kReanchorChunk +
                   sizeof(int) * ((size_t)8 * L.nshell * nsp * nsp + kReanchorChunk) +
                   (size_t)kReanchorChunk + (size_t)L.natoms;
        smem = std::max(smem, b);
        smem = std::max(smem, sizeof(int) * (size_t)L.ms_nblk);
    }
    CHX_REQUIRE(smem <= 200 * 1024, "reanchor: %zu bytes of shared memory needed", smem);
    CHX_REQUIRE(max_due > 0 && max_due <= nslots, "reanchor: max_due %d outside 1..%d", max_due,
                nslots);
    const int64_t need = ra_bytes(host_ladders, nladders, max_due);
    if (!scratch || scratch_bytes < need) {
        set_error("reanchor: scratch of %lld bytes needed, %lld given", (long long)need,
                  (long long)scratch_bytes);
        return CHX_ERR_SCRATCH;
    }
    const RaScratch R = ra_carve(scratch, max_due);
    const int nchunks = ra_nchunks(host_ladders, nladders);
    const int stride = (int)ra_partial_stride(host_ladders, nladders);
    const unsigned nitems = (unsigned)max_due * (unsigned)(nchunks + nsp);
    // a threshold picks up to max_due slots of the whole batch per call; a
    // mask (or every slot) is worked through in windows of max_due slots
    const int win = every > 0 ? nslots : max_due;
    for (int lo = 0; lo < nslots; lo += win) {
        const int hi = std::min(nslots, lo + win);
        k_reanchor_select<<<1, 1024, 0, st>>>(d_ladders, slot_ladder, lo, hi, mask, every,
                                              max_due, due, R, count);
        CHX_CHECK_LAUNCH("reanchor select");
#define CHX_RA(N)                                                                              \
    do {                                                                                       \
        cudaFuncSetAttribute(k_reanchor_part<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                             (int)smem);                                                       \
        k_reanchor_part<N><<<nitems, 256, smem, st>>>(d_ladders, slot_ladder, R, nchunks,      \
                                                      stride, d_err);                          \
        CHX_CHECK_LAUNCH("reanchor part");                                                     \
        k_reanchor_fin<N><<<max_due, 256, 0, st>>>(d_ladders, slot_ladder, R, nchunks, stride); \
    } while (0)
        switch (nsp) {
            case 2: CHX_RA(2); break;
            case 3: CHX_RA(3); break;
            case 4: CHX_RA(4); break;
            default: set_error("reanchor: nsp %d not built", nsp); return CHX_ERR_UNSUPPORTED;
        }
#undef CHX_RA
        CHX_CHECK_LAUNCH("reanchor fin");
    }
    return CHX_OK;
}

int64_t chx_reanchor_scratch_bytes(const chx_ladder_t *host_ladders, int nladders, int max_due) {
    if (!host_ladders || nladders <= 0 || max_due <= 0) return -1;
    return ra_bytes(host_ladders, nladders, std::min(max_due, kRaWindow));
}

int chx_refresh_chi2(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders,
                     int nladders, const int *slot_ladder, int nslots, int precision,
                     const uint8_t *mask, void *stream) {
    CHX_REQUIRE(d_ladders && host_ladders && slot_ladder && nladders > 0 && nslots > 0,
                "refresh_chi2: bad arguments");
    StepSmem so;
    size_t smem = 0;
    int rc = plan_ladders(host_ladders, nladders, precision, &so, &smem);
    if (rc != CHX_OK) return rc;
    cudaStream_t st = as_stream(stream);
    int nsp = host_ladders[0].nsp;
#define CHX_EV(N, PR) launch_eval<N, PR>(d_ladders, slot_ladder, nslots, so, smem, nullptr, nullptr, nullptr, mask, st)
    if (precision == CHX_FP64) {
        switch (nsp) {
            case 2: return CHX_EV(2, CHX_FP64);
            case 3: return CHX_EV(3, CHX_FP64);
            case 4: return CHX_EV(4, CHX_FP64);
        }
    } else {
        switch (nsp) {
            case 2: return CHX_EV(2, CHX_FP32C);
            case 3: return CHX_EV(3, CHX_FP32C);
            case 4: return CHX_EV(4, CHX_FP32C);
        }
    }
#undef CHX_EV
    set_error("refresh_chi2: nsp %d not built", nsp);
    return CHX_ERR_UNSUPPORTED;
}

int chx_reanchor(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders, int nladders,
                 const int *slot_ladder, int nslots, const uint8_t *mask, void *scratch,
                 int64_t scratch_bytes, int *d_err, void *stream) {
    CHX_REQUIRE(d_ladders && host_ladders && slot_ladder && d_err && nladders > 0 && nslots > 0,
                "reanchor: bad arguments");
    return reanchor_launch(d_ladders, host_ladders, nladders, slot_ladder, nslots, mask, 0,
                           std::min(nslots, kRaWindow), nullptr, nullptr, scratch, scratch_bytes,
                           d_err, as_stream(stream));
}

int chx_reanchor_due(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders,
                     int nladders, const int *slot_ladder, int nslots, int every, int max_due,
                     int precision, uint8_t *due, unsigned long long *count, void *scratch,
                     int64_t scratch_bytes, int *d_err, void *stream) {
    CHX_REQUIRE(d_ladders && host_ladders && slot_ladder && d_err && due && nladders > 0 &&
                    nslots > 0 && every > 0,
                "reanchor_due: bad arguments");
    cudaStream_t st = as_stream(stream);
    int rc = reanchor_launch(d_ladders, host_ladders, nladders, slot_ladder, nslots, nullptr,
                             every, max_due, due, count, scratch, scratch_bytes, d_err, st);
    if (rc != CHX_OK) return rc;
    StepSmem so;
    size_t smem = 0;
    rc = plan_ladders(host_ladders, nladders, precision, &so, &smem);
    if (rc != CHX_OK) return rc;
    int nsp = host_ladders[0].nsp;
#define CHX_EV(N, PR) launch_eval<N, PR>(d_ladders, slot_ladder, nslots, so, smem, nullptr, nullptr, nullptr, due, st)
    if (precision == CHX_FP64) {
        switch (nsp) {
            case 2: return CHX_EV(2, CHX_FP64);
            case 3: return CHX_EV(3, CHX_FP64);
            case 4: return CHX_EV(4, CHX_FP64);
        }
    } else {
        switch (nsp) {
            case 2: return CHX_EV(2, CHX_FP32C);
            case 3: return CHX_EV(3, CHX_FP32C);
            case 4: return CHX_EV(4, CHX_FP32C);
        }
    }
#undef CHX_EV
    set_error("reanchor_due: nsp %d not built", nsp);
    return CHX_ERR_UNSUPPORTED;
}

int chx_replica_exchange(const chx_ladder_t *d_ladders, int nladders, const uint64_t *round_key,
                         void *stream) {
    CHX_REQUIRE(d_ladders && round_key && nladders > 0, "replica_exchange: bad arguments");
    k_exchange<<<nladders, 128, 0, as_stream(stream)>>>(d_ladders, nladders, round_key);
    CHX_CHECK_LAUNCH("replica_exchange");
    return CHX_OK;
}

int chx_apply_exchange(const chx_ladder_t *d_ladders, int ladder, const int *order,
                       void *stream) {
    CHX_REQUIRE(d_ladders && order && ladder >= 0, "apply_exchange: bad arguments");
    k_apply_exchange<<<1, 32, 0, as_stream(stream)>>>(d_ladders, ladder, order);
    CHX_CHECK_LAUNCH("apply_exchange");
    return CHX_OK;
}

}  // extern "C"
