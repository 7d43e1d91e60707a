// chx_device.cuh -- device functions shared by the kernels of libchimera_b200.
#pragma once
#include "chx_common.cuh"

namespace chx {

// Proposal of one replica: draws exactly the reference's splitmix64 sequence
// (exafs_gpu/kernels.py:376-421) keyed (seed, step, replica index c).
struct Proposal {
    int a, b, nsa, nsb, swap;
    double np[3];
};

// The draws of one proposal that do not depend on the state: the move kind,
// site a and the eight candidate partners, keyed (seed, step, replica c).
// They can be drawn ahead of the step that uses them.
struct ProposalDraws {
    uint64_t h0;   // hash state after the draw of a (a displacement without swap)
    uint64_t h8;   // after the eight candidate draws (the failed swap's displacement)
    int sw, a;
    int cand[8];
};

__device__ __forceinline__ void propose_draws(ProposalDraws &d, uint64_t seed, uint64_t stepc,
                                              int c, int natoms, double swap_frac) {
    uint64_t h = splitmix64(seed ^ (stepc * 0x9E3779B97F4A7C15ULL) ^ ((uint64_t)c << 32));
    h = splitmix64(h);
    d.sw = (u01(h) < swap_frac) ? 1 : 0;
    h = splitmix64(h);
    int a = (int)(u01(h) * natoms);
    if (a >= natoms) a = natoms - 1;
    d.a = a;
    d.h0 = h;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        h = splitmix64(h);
        int cand = (int)(u01(h) * natoms);
        if (cand >= natoms) cand = natoms - 1;
        d.cand[t] = cand;
    }
    d.h8 = h;
}

// The proposal from its draws and the current species S(i) (an array or a
// shared-memory accessor): the first candidate of another species than a's
// is the swap partner; with none (or no swap drawn), a Gaussian displacement
// of a, Box-Muller on the draws that follow. keep_pos: also report a's
// position as np for a swap (the reference's proposal record); the fused
// step leaves it out, it reads np for displacements only.
template <typename SpeciesOf>
__device__ __forceinline__ Proposal propose_finish(const ProposalDraws &d, SpeciesOf S,
                                                   const double *P, const double *Id,
                                                   double disp_sigma, double max_disp,
                                                   bool keep_pos = true) {
    Proposal pr;
    const int a = d.a;
    int sa = S(a), b = a, sb = sa;
    if (d.sw) {
        for (int t = 0; t < 8; ++t) {
            int sc = S(d.cand[t]);
            if (sc != sa) {
                b = d.cand[t];
                sb = sc;
                break;
            }
        }
    }
    int real_swap = (d.sw && b != a) ? 1 : 0;
    pr.swap = real_swap;
    pr.a = a;
    pr.b = b;
    pr.nsa = real_swap ? sb : sa;
    pr.nsb = real_swap ? sa : sb;
    const double *Pa = P + (long)a * 3;
    const double *Ia = Id + (long)a * 3;
    if (real_swap) {
        if (keep_pos) {
            pr.np[0] = Pa[0];
            pr.np[1] = Pa[1];
            pr.np[2] = Pa[2];
        } else {
            pr.np[0] = pr.np[1] = pr.np[2] = 0.0;
        }
    } else {
        // a swap drawn but no partner found consumed all eight candidate draws
        uint64_t h = d.sw ? d.h8 : d.h0;
        // Box-Muller on two pairs of draws, clamped to max_disp from the site
        double g[3];
        for (int t = 0; t < 3; t += 2) {
            h = splitmix64(h);
            double u1 = u01(h);
            h = splitmix64(h);
            double u2 = u01(h);
            u1 = fmax(u1, 1e-300);
            double rad = sqrt(-2.0 * log(u1));
            g[t] = rad * cos(kTwoPi * u2);
            if (t + 1 < 3) g[t + 1] = rad * sin(kTwoPi * u2);
        }
        double ox = Pa[0] + g[0] * disp_sigma - Ia[0];
        double oy = Pa[1] + g[1] * disp_sigma - Ia[1];
        double oz = Pa[2] + g[2] * disp_sigma - Ia[2];
        double m = sqrt(ox * ox + oy * oy + oz * oz);
        double sc = (m > max_disp) ? (max_disp / m) : 1.0;
        pr.np[0] = Ia[0] + ox * sc;
        pr.np[1] = Ia[1] + oy * sc;
        pr.np[2] = Ia[2] + oz * sc;
    }
    return pr;
}

// Proposal of one replica: draws exactly the reference's splitmix64 sequence
// (exafs_gpu/kernels.py:376-421) keyed (seed, step, replica index c). The
// reference draws the candidates one at a time and stops at the first of
// another species; drawing all eight ahead reads the same stream, since a
// candidate draw after the partner is found is never used.
template <typename SpeciesOf>
__device__ __forceinline__ Proposal propose_one(SpeciesOf S, const double *P, const double *Id,
                                                int natoms, uint64_t seed, uint64_t stepc, int c,
                                                double swap_frac, double disp_sigma,
                                                double max_disp) {
    ProposalDraws d;
    propose_draws(d, seed, stepc, c, natoms, swap_frac);
    return propose_finish(d, S, P, Id, disp_sigma, max_disp);
}


// ------------------------------------------------------------- pair terms
// s02 f_b/(k r^2) exp(-2r/lam - 2k^2 s2) sin(2kr + delta_t - 4/3 k^3 C3),
// r = r + dr[shell][t] (exafs_gpu/kernels.py:22-29), FP64.
struct KPoint {
    double k, lam;
};

__device__ __forceinline__ double term64(double rr, int t, int sh, double s2, int ik, int nk,
                                         int nsp, const KPoint &kp, const double *ftab,
                                         const double *dtab, const double *drtab,
                                         const double *c3tab, const double *s2tab, double s02) {
    int nn = nsp * nsp;
    double re = rr + drtab[sh * nn + t];
    int sb = t % nsp;
    double amp = s02 * ftab[sb * nk + ik] / (kp.k * re * re) *
                 exp(-2.0 * re / kp.lam - 2.0 * kp.k * kp.k * (s2 + s2tab[sh * nn + t]));
    return amp * sin(2.0 * kp.k * re + dtab[t * nk + ik] -
                     (4.0 / 3.0) * kp.k * kp.k * kp.k * c3tab[sh]);
}


// 32-byte pair record: one directed pair of one configuration, folded with
// its per-(shell, type) offsets.
struct __align__(16) PairRec {
    double reff;   // r + dr[shell][t]
    double s2;     // sig2[p] + s2tab[shell][t]
    double c3;     // c3tab[shell]
    float inv_r2;  // 1 / reff^2
    int t;         // absorber * nsp + scatterer
};
static_assert(sizeof(PairRec) == 32, "pair record must be 32 bytes");

// Per-thread constants of one k point.
template <int NSP>
struct KConst {
    double k, twok, m2il, m2k2, c3k;  // k, 2k, -2/lam, -2k^2, 4/3 k^3
    double delta[NSP * NSP];
    double famp64[NSP];               // s02 f_b(k) / k
    float famp32[NSP];
};

template <int NSP>
__device__ __forceinline__ void load_kconst(KConst<NSP> &c, const double *ktab,
                                            const double *lamtab, const double *dtab,
                                            const double *ftab, double s02, int nk, int ik) {
    double k = ktab[ik], lam = lamtab[ik];
    c.k = k;
    c.twok = 2.0 * k;
    c.m2il = -2.0 / lam;
    c.m2k2 = -2.0 * k * k;
    c.c3k = (4.0 / 3.0) * k * k * k;
#pragma unroll
    for (int t = 0; t < NSP * NSP; ++t) c.delta[t] = dtab[t * nk + ik];
#pragma unroll
    for (int s = 0; s < NSP; ++s) {
        c.famp64[s] = s02 * ftab[s * nk + ik] / k;
        c.famp32[s] = (float)c.famp64[s];
    }
}

template <int NSP, int PREC>
__device__ __forceinline__ double rec_term(const PairRec &r, const KConst<NSP> &c) {
    int t = r.t;
    double dl = 0.0;
#pragma unroll
    for (int q = 0; q < NSP * NSP; ++q)
        if (q == t) dl = c.delta[q];
    double ph = fma(c.twok, r.reff, dl) - c.c3k * r.c3;
    double ex = fma(c.m2il, r.reff, c.m2k2 * r.s2);
    int sb = t % NSP;
    if (PREC == CHX_FP64) {
        double fa = 0.0;
#pragma unroll
        for (int q = 0; q < NSP; ++q)
            if (q == sb) fa = c.famp64[q];
        return fa / (r.reff * r.reff) * exp(ex) * sin(ph);
    } else {
        float fa = 0.0f;
#pragma unroll
        for (int q = 0; q < NSP; ++q)
            if (q == sb) fa = c.famp32[q];
        return (double)(fa * r.inv_r2 * expf((float)ex) * sinf(reduce_phase(ph)));
    }
}

}  // namespace chx
