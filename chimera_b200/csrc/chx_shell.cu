// chx_shell.cu -- the pair-count calibration objective for a population of
// parameter sets (chx_shell_rfactor).
//
// One CTA per member, FP64 throughout, in four barrier-separated phases:
//   1. chi_a(k) = sum_{b,s} N[a,b,s] B[a,b,s](k) / N_a + chi_MS,a(k) at the
//      member's parameters (chimera/shellmodel.py:290-336, 338-356, 411-413;
//      chimera/multiscat.py:133-145);
//   2. per channel (edge e, k weight w) the resampled, windowed row on the
//      uniform grid n dk: the member's k axis sqrt(k^2 - etok dE0[e])
//      (chimera/model.py:120-130), linear resampling, the Hanning window of
//      its kmin, kmax times k^w, zero off the model grid
//      (exafs_gpu/fourier.py:21-67);
//   3. the DFT of those rows on the fitted FFT bins from a table of the nfft
//      twiddles (e^{-2 pi i j / nfft}) in shared memory, times dk / sqrt(pi);
//   4. one amplitude per edge profiled out and the R-factor over all channels
//      (chimera/model.py:497-545), |chi(R)| for magnitude data.
// The sums of phases 3-4 run in a fixed order, so a member's result does not
// depend on the rest of the population.
#include "chx_common.cuh"

namespace chx {

constexpr int kShellThreads = 256;
constexpr double kShellDE0Cap = 200.0;   // |dE0| (eV) accepted per edge
constexpr double kShellPi = 3.141592653589793;

struct ShellPlan {
    int npar, nchan, ncap;                // ncap: uniform-grid taps 0 .. ncap-1
    size_t o_tw, o_chi, o_u, o_x, o_par, o_red, total;
};

// Taps 0 .. nfft/2 - 1 of the uniform grid: the transform uses the first
// half of the FFT grid, and a model k grid ending below (nfft/2 - 1) dk (51 A^-1
// for the reference's 2048 x 0.05) keeps every non-zero tap inside it.
static ShellPlan shell_plan(const chx_shell_t &S) {
    ShellPlan p;
    p.npar = chx_shell_nparam(S.nsp, S.nshell);
    p.nchan = S.nsp * S.nkw;
    p.ncap = S.nfft / 2;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t r = o; o += (bytes + 15) & ~(size_t)15; return r; };
    p.o_tw = take(sizeof(double2) * S.nfft);
    p.o_chi = take(sizeof(double) * S.nsp * S.nk);
    p.o_u = take(sizeof(double) * p.nchan * p.ncap);
    p.o_x = take(sizeof(double2) * p.nchan * S.nbin);
    p.o_par = take(sizeof(double) * p.npar);
    p.o_red = take(sizeof(double) * 4 * 16);
    p.total = o;
    return p;
}

__device__ __forceinline__ double hanning(double k, double kmin, double kmax, double dw) {
    // exafs_gpu/fourier.py:25-33: flat top, sine tapers of width dw
    double w = 0.0;
    if (k >= kmin + 0.5 * dw && k <= kmax - 0.5 * dw) w = 1.0;
    if (k > kmin - 0.5 * dw && k < kmin + 0.5 * dw)
        w = 0.5 * (1.0 + sin(kShellPi * (k - kmin) / dw));
    if (k > kmax - 0.5 * dw && k < kmax + 0.5 * dw)
        w = 0.5 * (1.0 - sin(kShellPi * (k - kmax) / dw));
    return w;
}

__global__ void __launch_bounds__(kShellThreads) k_shell_rfactor(chx_shell_t S, ShellPlan pl,
                                                                 const double *__restrict__ params,
                                                                 double *__restrict__ rf,
                                                                 double *__restrict__ scales) {
    extern __shared__ __align__(16) unsigned char smem[];
    double2 *tw = (double2 *)(smem + pl.o_tw);
    double *chi = (double *)(smem + pl.o_chi);
    double *u = (double *)(smem + pl.o_u);
    double2 *X = (double2 *)(smem + pl.o_x);
    double *par = (double *)(smem + pl.o_par);
    double *red = (double *)(smem + pl.o_red);
    __shared__ int s_bad;
    __shared__ int s_n0, s_n1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    const int m = blockIdx.x;
    const int nsp = S.nsp, nshell = S.nshell, nk = S.nk, nn = nsp * nsp;
    for (int q = tid; q < pl.npar; q += blockDim.x) par[q] = params[(long)m * pl.npar + q];
    for (int j = tid; j < S.nfft; j += blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)j / (double)S.nfft, &s, &c);
        tw[j] = make_double2(c, -s);
    }
    if (tid == 0) s_bad = 0;
    __syncthreads();
    const double a0 = par[0], sig_scale = par[1], ms_amp = par[2], ms_c = par[3];
    const double kmin = par[4], kmax = par[5];
    const double *dE0 = par + 6, *sss = dE0 + nsp, *dr = sss + nshell, *c3 = dr + nn,
                 *c4 = c3 + nshell, *spair = c4 + nshell, *ms_edge = spair + nn;
    const double rscale = a0 / S.a0_ref;
    const double *Nm = S.N_member ? S.N_member + (long)m * nsp * nsp * nshell : S.N;
    if (tid == 0) {
        double zsum = 0.0;
        for (int s = 0; s < nshell; ++s) zsum += S.shell_mult[s];
        red[60] = zsum;
        for (int e = 0; e < nsp; ++e) {
            if (!(fabs(dE0[e]) <= kShellDE0Cap)) s_bad = 1;      // also catches NaN
            const double kk = S.k[nk - 1];
            if (sqrt(fmax(kk * kk - S.etok * dE0[e], 1e-4)) > (pl.ncap - 1) * S.dk) s_bad = 1;
        }
        if (!(isfinite(kmin) && isfinite(kmax) && isfinite(a0) && a0 > 0.0)) s_bad = 1;
        const double lo = kmin - 0.5 * S.dk_win, hi = kmax + 0.5 * S.dk_win;
        const double top = (double)(pl.ncap - 1);
        // clamped in FP64 first, so no out-of-range value reaches the int casts
        s_n0 = s_bad ? 0 : (int)fmin(fmax(floor(lo / S.dk), 0.0), top);
        s_n1 = s_bad ? -1 : (int)fmin(fmax(ceil(hi / S.dk), -1.0), top);
    }
    __syncthreads();
    const double zsum = red[60];

    // ---- 1. chi_a(k) at the member's parameters
    const double r_nn = S.shells_ref[0] * rscale;
    const double s2nn = S.sigma2_ref[0] * sig_scale * sss[0];
    for (int it = tid; it < nsp * nk; it += blockDim.x) {
        const int a = it / nk, ik = it - a * nk;
        const double k = S.k[ik], k2 = k * k, k3 = k2 * k, k4 = k2 * k2;
        const double lam = S.lam[ik];
        double acc = 0.0, cnt = 0.0;
        for (int s = 0; s < nshell; ++s) {
            const double rs = S.shells_ref[s] * rscale;
            const double s2 = S.sigma2_ref[s] * sig_scale * sss[s];
            const double amp4 = (2.0 / 3.0) * k4 * c4[s];
            const double ph3 = (4.0 / 3.0) * k3 * c3[s];
            for (int b = 0; b < nsp; ++b) {
                const double Nab = Nm[(a * nsp + b) * nshell + s];
                cnt += Nab;
                if (Nab == 0.0) continue;
                const double r = rs + (s == 0 ? dr[a * nsp + b] : 0.0);
                const double s2ab = s2 * (s == 0 ? spair[a * nsp + b] : 1.0);
                const double B = S.s02 * S.f[b * nk + ik] / (k * r * r) *
                                 exp(-2.0 * r / lam - 2.0 * k2 * s2ab + amp4) *
                                 sin(2.0 * k * r + S.delta[(a * nsp + b) * nk + ik] - ph3);
                acc += Nab * B;
            }
        }
        double v = acc / fmax(cnt / zsum, 1e-30);
        if (S.npath > 0) {
            const double ascale = r_nn / S.ms_dnn;
            double ms = 0.0;
            for (int q = 0; q < S.npath; ++q) {
                if (S.ms_abs[q] != a) continue;
                const double r = S.ms_reff[q] * ascale;
                const double s2 = ms_c * s2nn * r / (2.0 * r_nn);
                const long o = (long)q * nk + ik;
                ms += S.ms_deg[q] * S.s02 * S.ms_F[o] / fmax(k * r * r, 1e-12) *
                      exp(-2.0 * r / fmax(S.ms_L[o], 1e-6) - 2.0 * k2 * s2) *
                      sin(2.0 * k * r + S.ms_D[o]);
            }
            v += ms_amp * ms * ms_edge[a];
        }
        chi[it] = v;
    }
    __syncthreads();

    // ---- 2. resampled, windowed rows on the uniform grid (taps n0 .. n1)
    const int n0 = s_n0, n1 = s_n1, ntap = n1 - n0 + 1;
    for (int it = tid; it < pl.nchan * ntap; it += blockDim.x) {
        const int c = it / ntap, n = n0 + (it - c * ntap);
        const int e = c / S.nkw, w = S.kweight[c - e * S.nkw];
        const double ku = (double)n * S.dk;
        const double shift = S.etok * dE0[e];
        auto kmod = [&](int i) { double kk = S.k[i]; return sqrt(fmax(kk * kk - shift, 1e-4)); };
        const double kfirst = kmod(0), klast = kmod(nk - 1);
        double val = 0.0;
        if (ku >= kfirst && ku <= klast) {
            double win = hanning(ku, kmin, kmax, S.dk_win);
            if (win != 0.0) {
                // first i with kmod(i) >= ku, minus one (searchsorted, left)
                int lo = 0, hi = nk;
                while (lo < hi) {
                    int mid = (lo + hi) >> 1;
                    if (kmod(mid) < ku) lo = mid + 1;
                    else hi = mid;
                }
                int idx = min(max(lo - 1, 0), nk - 2);
                const double ka = kmod(idx), kb = kmod(idx + 1);
                const double span = fmax(kb - ka, 1e-12);
                const double frac = fmin(fmax((ku - ka) / span, 0.0), 1.0);
                const double ca = chi[e * nk + idx], cb = chi[e * nk + idx + 1];
                double kw = 1.0;
                for (int q = 0; q < w; ++q) kw *= ku;
                val = (ca + (cb - ca) * frac) * (win * kw);
            }
        }
        u[c * pl.ncap + n] = val;
    }
    __syncthreads();

    // ---- 3. DFT on the fitted bins
    const double norm = S.dk / sqrt(kShellPi);
    const int fmask = S.nfft - 1;
    for (int it = tid; it < pl.nchan * S.nbin; it += blockDim.x) {
        const int c = it / S.nbin, q = it - c * S.nbin;
        const int bin = S.bins[q];
        const double *uc = u + c * pl.ncap;
        double re = 0.0, im = 0.0;
        for (int n = n0; n <= n1; ++n) {
            const double x = uc[n];
            const double2 t = tw[(int)(((long)n * bin) & fmask)];
            re = fma(x, t.x, re);
            im = fma(x, t.y, im);
        }
        re *= norm;
        im *= norm;
        if (S.magnitude) {
            re = sqrt(re * re + im * im);
            im = 0.0;
        }
        X[it] = make_double2(re, im);
    }
    __syncthreads();

    // ---- 4. per-channel sums, one amplitude per edge, the R-factor
    double *num = red, *den = red + 16, *dd = red + 32, *res = red + 48;
    for (int c = warp; c < pl.nchan; c += nwarp) {
        double a_ = 0.0, b_ = 0.0, d_ = 0.0;
        for (int q = lane; q < S.nbin; q += 32) {
            const double2 x = X[c * S.nbin + q];
            const double dr_ = S.data[((long)c * S.nbin + q) * 2];
            const double di_ = S.magnitude ? 0.0 : S.data[((long)c * S.nbin + q) * 2 + 1];
            a_ += x.x * dr_ + x.y * di_;
            b_ += x.x * x.x + x.y * x.y;
            d_ += dr_ * dr_ + di_ * di_;
        }
        a_ = warp_sum(a_);
        b_ = warp_sum(b_);
        d_ = warp_sum(d_);
        if (lane == 0) {
            num[c] = a_;
            den[c] = b_;
            dd[c] = d_;
        }
    }
    __syncthreads();
    __shared__ double s_scale[16];
    if (tid == 0) {
        for (int e = 0; e < nsp; ++e) {
            double nu = 0.0, de = 0.0;
            for (int q = 0; q < S.nkw; ++q) {
                nu += num[e * S.nkw + q];
                de += den[e * S.nkw + q];
            }
            s_scale[e] = S.profile ? nu / fmax(de, 1e-30) : 1.0;
        }
    }
    __syncthreads();
    for (int c = warp; c < pl.nchan; c += nwarp) {
        const double sc = s_scale[c / S.nkw];
        double r_ = 0.0;
        for (int q = lane; q < S.nbin; q += 32) {
            const double2 x = X[c * S.nbin + q];
            const double dr_ = S.data[((long)c * S.nbin + q) * 2];
            const double di_ = S.magnitude ? 0.0 : S.data[((long)c * S.nbin + q) * 2 + 1];
            const double er = sc * x.x - dr_, ei = sc * x.y - di_;
            r_ += er * er + ei * ei;
            if (S.resid) {
                const double sg = S.sigma ? S.sigma[(long)c * S.nbin + q] : 1.0;
                double *o = S.resid + (((long)m * pl.nchan + c) * S.nbin + q) * 2;
                o[0] = er / sg;
                o[1] = ei / sg;
            }
        }
        r_ = warp_sum(r_);
        if (lane == 0) res[c] = r_;
    }
    __syncthreads();
    if (tid == 0) {
        double tn = 0.0, td = 0.0;
        for (int c = 0; c < pl.nchan; ++c) {
            tn += res[c];
            td += dd[c];
        }
        rf[m] = s_bad ? nan("") : tn / fmax(td, 1e-30);
        for (int e = 0; e < nsp; ++e) scales[(long)m * nsp + e] = s_bad ? nan("") : s_scale[e];
    }
}

}  // namespace chx

using namespace chx;

extern "C" {

int chx_shell_nparam(int nsp, int nshell) {
    if (nsp <= 0 || nshell <= 0) return -1;
    return 6 + nsp + nshell + nsp * nsp + 2 * nshell + nsp * nsp + nsp;
}

int chx_shell_rfactor(const chx_shell_t *S, const double *params, int P, double *rf,
                      double *scales, void *stream) {
    CHX_REQUIRE(S && params && rf && scales && P > 0, "shell_rfactor: bad arguments");
    CHX_REQUIRE(S->nsp >= 1 && S->nsp <= 4 && S->nshell >= 1 && S->nk >= 2 && S->nkw >= 1 &&
                    S->nsp * S->nkw <= 16 && S->nbin >= 1 && S->nfft >= 2 &&
                    (S->nfft & (S->nfft - 1)) == 0 && S->dk > 0.0 && S->dk_win > 0.0,
                "shell_rfactor: sizes outside the built limits (nsp %d, nkw %d, nbin %d, nfft %d)",
                S->nsp, S->nkw, S->nbin, S->nfft);
    CHX_REQUIRE(S->k && S->f && S->delta && S->lam && S->shells_ref && S->sigma2_ref &&
                    S->shell_mult && (S->N || S->N_member) && S->kweight && S->bins && S->data,
                "shell_rfactor: a model array is NULL");
    CHX_REQUIRE(S->npath == 0 || (S->ms_abs && S->ms_reff && S->ms_deg && S->ms_F && S->ms_D &&
                                  S->ms_L && S->ms_dnn > 0.0),
                "shell_rfactor: incomplete multiple-scattering paths");
    ShellPlan pl = shell_plan(*S);
    CHX_REQUIRE(pl.total <= 227 * 1024, "shell_rfactor: %zu bytes of shared memory needed",
                pl.total);
    cudaError_t e = cudaFuncSetAttribute(k_shell_rfactor, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)pl.total);
    if (e != cudaSuccess) return cuda_fail(e, "shell_rfactor: shared memory attribute");
    k_shell_rfactor<<<P, kShellThreads, pl.total, as_stream(stream)>>>(*S, pl, params, rf,
                                                                      scales);
    CHX_CHECK_LAUNCH("shell_rfactor");
    return CHX_OK;
}

}  // extern "C"
