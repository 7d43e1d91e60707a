// chx_path.cu -- curved-wave multiple-scattering path trace (chx_path_trace).
//
// Tr_{l=1} of the path product P = G(a_N) t_N D_N ... t_1 D_1 G(a_0), then the
// closing rotation, for a K edge (exafs_gpu/abinitio/pathsum.py:1-22,
// 106-126): three state columns (the l = 1, mu = -1, 0, 1 start vectors) of
// (lmax+1)^2 complex amplitudes each, in every leg's own frame. One CTA per
// (energy, path), FP64 complex; the state is ping-ponged between two
// shared-memory buffers, one barrier per pass:
//   t:        v_lm *= t_l(type)
//   rotation: x = i^{-m} e^{-i m gamma} v; y_m'' = e^{-i m'' beta} sum_m' Delta_{m''m'} x_m';
//             w_m = i^m e^{-i m alpha} sum_m'' Delta_{m''m} y_m''   (Delta = d^l(pi/2))
//   leg:      w_l'm = sum_l g^m_{l'l}(p |a|) v_lm,  g = sum_l'' A^m_{l'l l''} h_l''(p |a|),
//             one |m| block of g built in shared memory and applied to +-m,
//             h by upward recurrence from h_0 = -i e^{ix}/x, h_1 = -e^{ix}/x (1 + i/x).
#include "chx_common.cuh"

namespace chx {

constexpr int kPathThreads = 256;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) {
    return make_double2(a.x * s, a.y * s);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
// i^n for an integer n
__device__ __forceinline__ double2 ipow(int n) {
    n &= 3;
    return n == 0 ? make_double2(1, 0) : n == 1 ? make_double2(0, 1)
                 : n == 2 ? make_double2(-1, 0) : make_double2(0, -1);
}
// e^{-i m a}
__device__ __forceinline__ double2 phase(int m, double a) {
    double s, c;
    sincos(-(double)m * a, &s, &c);
    return make_double2(c, s);
}
__device__ __forceinline__ int l_of(int L) {
    int l = (int)sqrtf((float)L + 0.5f);
    while (l * l > L) --l;
    while ((l + 1) * (l + 1) <= L) ++l;
    return l;
}

__global__ void __launch_bounds__(kPathThreads) k_path_trace(chx_path_t P, double *__restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int G = P.glmax, NLM = (G + 1) * (G + 1);
    double2 *bufA = (double2 *)smem, *bufB = bufA + 3 * NLM, *hk = bufB + 3 * NLM;
    double2 *gb = hk + 2 * G + 2;                   // (G+1)^2: one |m| block of g
    const int ie = blockIdx.x, ip = blockIdx.y, tid = threadIdx.x, nth = blockDim.x;
    const int ns = P.nsc[ip];
    const int lm = P.lmax[(long)ip * P.ne + ie];
    double *o = out + ((long)ip * P.ne + ie) * 2;
    // uniform over the CTA: every thread reads the same values
    if (ns < 0 || ns > P.maxs || lm < 1 || lm > G) {
        if (tid == 0) o[0] = o[1] = nan("");
        return;
    }
    for (int j = 0; j < ns; ++j) {
        const int ty = P.typ[(long)ip * P.maxs + j];
        if (ty < 0 || ty >= P.ntype) {
            if (tid == 0) o[0] = o[1] = nan("");
            return;
        }
    }
    const int nlm = (lm + 1) * (lm + 1);
    const double2 p = make_double2(P.p[2 * ie], P.p[2 * ie + 1]);
    double2 *v = bufA, *w = bufB;
    for (int q = tid; q < 3 * NLM; q += nth) v[q] = make_double2(0, 0);
    __syncthreads();
    if (tid < 3) v[tid * NLM + 2 + (tid - 1)] = make_double2(1, 0);   // (l, m) = (1, tid-1)
    __syncthreads();

    for (int j = 0; j <= ns; ++j) {
        if (j > 0) {
            // ---- scatterer j: t_l, then the rotation into leg j's frame
            const int ty = P.typ[(long)ip * P.maxs + j - 1];
            const double *t = P.t + (((long)ty * P.ne + ie) * P.nlt) * 2;
            const double *e = P.eul + ((long)ip * (P.maxs + 1) + (j - 1)) * 3;
            const double al = e[0], be = e[1], ga = e[2];
            for (int q = tid; q < 3 * nlm; q += nth) {
                const int c = q / nlm, L = q - c * nlm;
                const int l = l_of(L), m = L - l * l - l;
                const double2 tv = make_double2(t[2 * l], t[2 * l + 1]);
                v[c * NLM + L] = cmul(cmul(v[c * NLM + L], tv), cmul(ipow(-m), phase(m, ga)));
            }
            __syncthreads();
            for (int q = tid; q < 3 * nlm; q += nth) {
                const int c = q / nlm, L = q - c * nlm;
                const int l = l_of(L), mpp = L - l * l - l;
                const double *D = P.dflat + P.doff[l] + (long)(mpp + l) * (2 * l + 1);
                double2 acc = make_double2(0, 0);
                for (int mp = -l; mp <= l; ++mp)
                    acc = cadd(acc, cscale(v[c * NLM + l * l + l + mp], D[mp + l]));
                w[c * NLM + L] = cmul(acc, phase(mpp, be));
            }
            __syncthreads();
            { double2 *s = v; v = w; w = s; }
            for (int q = tid; q < 3 * nlm; q += nth) {
                const int c = q / nlm, L = q - c * nlm;
                const int l = l_of(L), m = L - l * l - l;
                const double *D = P.dflat + P.doff[l];
                double2 acc = make_double2(0, 0);
                for (int mpp = -l; mpp <= l; ++mpp)
                    acc = cadd(acc, cscale(v[c * NLM + l * l + l + mpp],
                                           D[(long)(mpp + l) * (2 * l + 1) + (m + l)]));
                w[c * NLM + L] = cmul(acc, cmul(ipow(m), phase(m, al)));
            }
            __syncthreads();
            { double2 *s = v; v = w; w = s; }
        }
        // ---- leg j: Hankel functions h_0 .. h_{2 lm}(p |a_j|), then the propagator
        if (tid == 0) {
            const double R = P.leg[(long)ip * (P.maxs + 1) + j];
            const double2 x = cscale(p, R);
            double s, c;
            sincos(x.x, &s, &c);
            const double2 ex = cscale(make_double2(c, s), exp(-x.y));     // e^{i x}
            hk[0] = cdiv(cmul(make_double2(0, -1), ex), x);
            hk[1] = cmul(cscale(cdiv(ex, x), -1.0), cadd(make_double2(1, 0),
                                                         cdiv(make_double2(0, 1), x)));
            for (int l = 1; l < 2 * lm; ++l)
                hk[l + 1] = cadd(cdiv(cscale(hk[l], (double)(2 * l + 1)), x),
                                 cscale(hk[l - 1], -1.0));
        }
        __syncthreads();
        // one |m| block at a time: g^|m|_{l'l} (l', l = |m| .. lm) built once
        // into shared memory, then applied to m = +|m| and -|m| of all three
        // columns (g is even in m)
        for (int am = 0; am <= lm; ++am) {
            const int n = lm - am + 1;
            for (int q = tid; q < n * n; q += nth) {
                const int lp = am + q / n, l = am + (q - (q / n) * n);
                const long g3 = ((long)am * (G + 1) + lp) * (G + 1) + l;
                const int off = P.goff[g3], cnt = P.gcnt[g3];
                double2 g = make_double2(0, 0);
                for (int u = 0; u < cnt; ++u) {
                    const double2 A = make_double2(P.gA[2 * (off + u)], P.gA[2 * (off + u) + 1]);
                    g = cadd(g, cmul(A, hk[P.glpp[off + u]]));
                }
                gb[q] = g;
            }
            __syncthreads();
            const int nsg = am ? 2 : 1;
            for (int q = tid; q < 3 * nsg * n; q += nth) {
                const int c = q / (nsg * n), r = q - c * (nsg * n);
                const int m = (r / n) ? -am : am, lp = am + (r - (r / n) * n);
                const double2 *grow = gb + (lp - am) * n;
                double2 acc = make_double2(0, 0);
                for (int l = am; l <= lm; ++l)
                    acc = cadd(acc, cmul(grow[l - am], v[c * NLM + l * l + l + m]));
                w[c * NLM + lp * lp + lp + m] = acc;
            }
            __syncthreads();
        }
        { double2 *s = v; v = w; w = s; }
    }
    // ---- closing rotation, l = 1 rows only, and the trace
    if (tid == 0) {
        const double *e = P.eul + ((long)ip * (P.maxs + 1) + ns) * 3;
        const double al = e[0], be = e[1], ga = e[2];
        const double *D = P.dflat + P.doff[1];
        double2 tr = make_double2(0, 0);
        for (int c = 0; c < 3; ++c) {
            const int mu = c - 1;
            for (int mp = -1; mp <= 1; ++mp) {
                double2 d = make_double2(0, 0);          // d^1_{mu mp}(beta)
                for (int mpp = -1; mpp <= 1; ++mpp)
                    d = cadd(d, cscale(phase(mpp, be), D[(mpp + 1) * 3 + (mu + 1)] *
                                                           D[(mpp + 1) * 3 + (mp + 1)]));
                d = cmul(d, ipow(mu - mp));
                const double2 Dm = cmul(cmul(phase(mu, al), d), phase(mp, ga));
                tr = cadd(tr, cmul(Dm, v[c * NLM + 2 + mp]));
            }
        }
        o[0] = tr.x;
        o[1] = tr.y;
    }
}

}  // namespace chx

using namespace chx;

extern "C" {

int chx_path_trace(const chx_path_t *P, double *out, void *stream) {
    CHX_REQUIRE(P && out && P->npath > 0 && P->ne > 0 && P->maxs >= 1 && P->ntype >= 1 &&
                    P->glmax >= 1 && P->glmax <= 40 && P->nlt >= P->glmax + 1,
                "path_trace: bad sizes (npath %d, ne %d, maxs %d, glmax %d, nlt %d)",
                P ? P->npath : 0, P ? P->ne : 0, P ? P->maxs : 0, P ? P->glmax : 0,
                P ? P->nlt : 0);
    CHX_REQUIRE(P->nsc && P->typ && P->leg && P->eul && P->p && P->t && P->lmax && P->goff &&
                    P->gcnt && P->glpp && P->gA && P->doff && P->dflat,
                "path_trace: an array is NULL");
    CHX_REQUIRE(P->npath <= 65535, "path_trace: at most 65535 paths per call");
    const size_t nlm = (size_t)(P->glmax + 1) * (P->glmax + 1);
    const size_t smem = sizeof(double2) * (7 * nlm + 2 * (size_t)P->glmax + 2);
    CHX_REQUIRE(smem <= 227 * 1024, "path_trace: %zu bytes of shared memory needed", smem);
    cudaError_t e = cudaFuncSetAttribute(k_path_trace, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "path_trace: shared memory attribute");
    dim3 grid(P->ne, P->npath);
    k_path_trace<<<grid, kPathThreads, smem, as_stream(stream)>>>(*P, out);
    CHX_CHECK_LAUNCH("path_trace");
    return CHX_OK;
}

}  // extern "C"
