/*
 * chx_oracle.c -- CPU restatement of the reference's hot-path kernels.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker: only tests/, the
 * smoke() entry and bench.py's cpu_baseline / --impl reference legs load it.
 * Nothing in the chimera_b200 package links or calls it.
 *
 * Every function restates one reference kernel or method in plain C, FP64,
 * single-threaded, in the reference's own argument order and meaning:
 *
 *   orc_compute_r        exafs_gpu/kernels.py:53-78
 *   orc_build_ptype      exafs_gpu/kernels.py:81-96
 *   orc_chi_forward      exafs_gpu/kernels.py:99-163 (pair term :22-26)
 *   orc_chi_delta        exafs_gpu/kernels.py:243-325
 *   orc_commit_move      exafs_gpu/kernels.py:328-346
 *   orc_splitmix64/u01   exafs_gpu/kernels.py:352-360
 *   orc_propose_select   exafs_gpu/kernels.py:362-423
 *   orc_propose_build    exafs_gpu/kernels.py:425-488
 *   orc_commit_state     exafs_gpu/kernels.py:490-511
 *   orc_ms_counts        chimera/mslibrary.py:420-451 (entry code :433-434)
 *   orc_ms_delta         chimera/mslibrary.py:466-486
 *   orc_ft_window        exafs_gpu/fourier.py:69-80 evaluated as a direct DFT
 *                        on the requested R bins (the reference runs an FFT of
 *                        length nfft and slices; the sums are the same)
 *   orc_chi2             methods/method_a_rmc.py:190-227
 *
 * Sums run sequentially; the reference reduces over 256 threads, so the two
 * agree to FP64 rounding, not bit for bit. Integer outputs are exact.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_TWO_PI 6.283185307179586

/* ------------------------------------------------------------ geometry */
void orc_compute_r(const double *pos, const int *iidx, const int *jidx,
                   const double *shift, double *r, double *evec,
                   int npairs, int natoms, int nconf)
{
    for (int ic = 0; ic < nconf; ++ic)
        for (int p = 0; p < npairs; ++p) {
            long tid = (long)ic * npairs + p;
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
}

void orc_build_ptype(const int *species, const int *iidx, const int *jidx,
                     int *ptype, int npairs, int natoms, int nconf, int nsp)
{
    for (int ic = 0; ic < nconf; ++ic)
        for (int p = 0; p < npairs; ++p) {
            int sa = species[(long)ic * natoms + iidx[p]];
            int sb = species[(long)ic * natoms + jidx[p]];
            ptype[(long)ic * npairs + p] = sa * nsp + sb;
        }
}

/* One single-scattering pair term at one k point (kernels.py:22-26). */
static inline double orc_term(double rr, int t, int sh, int ik, int nk, int nsp,
                              double s2, double kv, double lam,
                              const double *ftab, const double *dtab,
                              const double *drtab, const double *c3tab,
                              const double *s2tab, double s02)
{
    int nn = nsp * nsp;
    double r_eff = rr + drtab[sh * nn + t];
    int sb = t % nsp;
    double amp = s02 * ftab[sb * nk + ik] / (kv * r_eff * r_eff)
               * exp(-2.0 * r_eff / lam - 2.0 * kv * kv * (s2 + s2tab[sh * nn + t]));
    return amp * sin(2.0 * kv * r_eff + dtab[t * nk + ik]
                     - (4.0 / 3.0) * kv * kv * kv * c3tab[sh]);
}

void orc_chi_forward(const double *r, const int *ptype, const int *shell,
                     const double *sig2, const double *ftab, const double *dtab,
                     const double *lamtab, const double *ktab, const double *drtab,
                     const double *c3tab, const double *s2tab, double *chi,
                     int npairs, int nk, int nconf, double s02, int nsp)
{
    double *acc = (double *)calloc((size_t)nsp, sizeof(double));
    for (int ic = 0; ic < nconf; ++ic)
        for (int ik = 0; ik < nk; ++ik) {
            memset(acc, 0, sizeof(double) * nsp);
            double kv = ktab[ik], lam = lamtab[ik];
            for (int p = 0; p < npairs; ++p) {
                int t = ptype[(long)ic * npairs + p];
                double v = orc_term(r[(long)ic * npairs + p], t, shell[p], ik, nk, nsp,
                                    sig2[p], kv, lam, ftab, dtab, drtab, c3tab, s2tab, s02);
                acc[t / nsp] += v;
            }
            for (int a = 0; a < nsp; ++a)
                chi[((long)ic * nsp + a) * nk + ik] = acc[a];
        }
    free(acc);
}

void orc_chi_delta(const double *r_old, const int *pt_old, const int *shell,
                   const int *aff, const double *r_new, const int *pt_new,
                   const double *sig2, const double *ftab, const double *dtab,
                   const double *lamtab, const double *ktab, const double *drtab,
                   const double *c3tab, const double *s2tab, double *dchi,
                   int npairs, int nk, int nrep, int maxaff, double s02, int nsp)
{
    double *acc = (double *)calloc((size_t)nsp, sizeof(double));
    for (int ic = 0; ic < nrep; ++ic)
        for (int ik = 0; ik < nk; ++ik) {
            memset(acc, 0, sizeof(double) * nsp);
            double kv = ktab[ik], lam = lamtab[ik];
            for (int q = 0; q < maxaff; ++q) {
                int p = aff[(long)ic * maxaff + q];
                if (p < 0) continue;
                int t = pt_new[(long)ic * maxaff + q];
                acc[t / nsp] += orc_term(r_new[(long)ic * maxaff + q], t, shell[p], ik, nk,
                                         nsp, sig2[p], kv, lam, ftab, dtab, drtab, c3tab,
                                         s2tab, s02);
                t = pt_old[(long)ic * npairs + p];
                acc[t / nsp] -= orc_term(r_old[(long)ic * npairs + p], t, shell[p], ik, nk,
                                         nsp, sig2[p], kv, lam, ftab, dtab, drtab, c3tab,
                                         s2tab, s02);
            }
            for (int a = 0; a < nsp; ++a)
                dchi[((long)ic * nsp + a) * nk + ik] = acc[a];
        }
    free(acc);
}

void orc_commit_move(const int *aff, const double *r_new, const int *pt_new,
                     const unsigned char *accept, double *r_old, int *pt_old,
                     int npairs, int nrep, int maxaff)
{
    for (int ic = 0; ic < nrep; ++ic) {
        if (!accept[ic]) continue;
        for (int q = 0; q < maxaff; ++q) {
            int p = aff[(long)ic * maxaff + q];
            if (p < 0) continue;
            r_old[(long)ic * npairs + p] = r_new[(long)ic * maxaff + q];
            pt_old[(long)ic * npairs + p] = pt_new[(long)ic * maxaff + q];
        }
    }
}

/* ------------------------------------------------------------ proposals */
uint64_t orc_splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

double orc_u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

void orc_propose_select(const int *species, const double *pos, const double *ideal,
                        int *a_out, int *b_out, int *newsa, int *newsb,
                        double *newpa, unsigned char *isswap,
                        int natoms, int nrep, uint64_t seed, uint64_t stepc,
                        double swap_frac, double disp_sigma, double max_disp)
{
    for (int c = 0; c < nrep; ++c) {
        uint64_t h = orc_splitmix64(seed ^ (stepc * 0x9E3779B97F4A7C15ULL)
                                    ^ ((uint64_t)c << 32));
        h = orc_splitmix64(h);
        int sw = (orc_u01(h) < swap_frac) ? 1 : 0;
        h = orc_splitmix64(h);
        int a = (int)(orc_u01(h) * natoms);
        if (a >= natoms) a = natoms - 1;
        const int *S = species + (long)c * natoms;
        int sa = S[a], b = a, sb = sa;
        if (sw) {
            for (int t = 0; t < 8; ++t) {
                h = orc_splitmix64(h);
                int cand = (int)(orc_u01(h) * natoms);
                if (cand >= natoms) cand = natoms - 1;
                if (S[cand] != sa) { b = cand; sb = S[cand]; break; }
            }
        }
        int real_swap = (sw && b != a) ? 1 : 0;
        isswap[c] = (unsigned char)real_swap;
        a_out[c] = a;
        b_out[c] = b;
        newsa[c] = real_swap ? sb : sa;
        newsb[c] = real_swap ? sa : sb;
        const double *P = pos + ((long)c * natoms + a) * 3;
        const double *Id = ideal + ((long)c * natoms + a) * 3;
        double np3[3];
        if (real_swap) {
            np3[0] = P[0]; np3[1] = P[1]; np3[2] = P[2];
        } else {
            double g[3];
            for (int t = 0; t < 3; t += 2) {
                h = orc_splitmix64(h); double u1 = orc_u01(h);
                h = orc_splitmix64(h); double u2 = orc_u01(h);
                u1 = fmax(u1, 1e-300);
                double rad = sqrt(-2.0 * log(u1));
                g[t] = rad * cos(ORC_TWO_PI * u2);
                if (t + 1 < 3) g[t + 1] = rad * sin(ORC_TWO_PI * u2);
            }
            double ox = P[0] + g[0] * disp_sigma - Id[0];
            double oy = P[1] + g[1] * disp_sigma - Id[1];
            double oz = P[2] + g[2] * disp_sigma - Id[2];
            double m = sqrt(ox * ox + oy * oy + oz * oz);
            double sc = (m > max_disp) ? (max_disp / m) : 1.0;
            np3[0] = Id[0] + ox * sc; np3[1] = Id[1] + oy * sc; np3[2] = Id[2] + oz * sc;
        }
        newpa[3 * c] = np3[0]; newpa[3 * c + 1] = np3[1]; newpa[3 * c + 2] = np3[2];
    }
}

void orc_propose_build(const int *species, const double *pos, const int *nbr,
                       const int *rev, const int *iidx, const int *jidx,
                       const double *shift, const int *a_in, const int *b_in,
                       const int *newsa, const int *newsb, const double *newpa,
                       int *aff, double *r_new, int *pt_new,
                       int natoms, int ncoord, int npairs, int nrep, int maxaff, int nsp)
{
    (void)npairs;
    for (int c = 0; c < nrep; ++c)
        for (int q = 0; q < maxaff; ++q) {
            long tid = (long)c * maxaff + q;
            int a = a_in[c], b = b_in[c];
            int blk = q / ncoord, o = q % ncoord;
            int p;
            if (blk == 0) p = nbr[(long)a * ncoord + o];
            else if (blk == 1) p = rev[nbr[(long)a * ncoord + o]];
            else if (blk == 2) p = nbr[(long)b * ncoord + o];
            else p = rev[nbr[(long)b * ncoord + o]];
            if (blk >= 2) {
                if (b == a) p = -1;
                else {
                    int other = (blk == 2) ? jidx[p] : iidx[p];
                    if (other == a) p = -1;
                }
            }
            aff[tid] = p;
            if (p < 0) { r_new[tid] = 0.0; pt_new[tid] = 0; continue; }
            int i = iidx[p], j = jidx[p];
            const double *P = pos + (long)c * natoms * 3;
            const double *NP = newpa + 3 * c;
            double pix, piy, piz, pjx, pjy, pjz;
            if (i == a) { pix = NP[0]; piy = NP[1]; piz = NP[2]; }
            else { pix = P[3 * i]; piy = P[3 * i + 1]; piz = P[3 * i + 2]; }
            if (j == a) { pjx = NP[0]; pjy = NP[1]; pjz = NP[2]; }
            else { pjx = P[3 * j]; pjy = P[3 * j + 1]; pjz = P[3 * j + 2]; }
            double dx = pjx + shift[3 * p + 0] - pix;
            double dy = pjy + shift[3 * p + 1] - piy;
            double dz = pjz + shift[3 * p + 2] - piz;
            r_new[tid] = sqrt(dx * dx + dy * dy + dz * dz);
            const int *S = species + (long)c * natoms;
            int si = (i == a) ? newsa[c] : ((i == b) ? newsb[c] : S[i]);
            int sj = (j == a) ? newsa[c] : ((j == b) ? newsb[c] : S[j]);
            pt_new[tid] = si * nsp + sj;
        }
}

void orc_commit_state(const unsigned char *accept, const int *a_in, const int *b_in,
                      const int *newsa, const int *newsb, const double *newpa,
                      const unsigned char *isswap, int *species, double *pos,
                      int natoms, int nrep)
{
    for (int c = 0; c < nrep; ++c) {
        if (!accept[c]) continue;
        int a = a_in[c], b = b_in[c];
        species[(long)c * natoms + a] = newsa[c];
        species[(long)c * natoms + b] = newsb[c];
        if (!isswap[c]) {
            double *P = pos + ((long)c * natoms + a) * 3;
            P[0] = newpa[3 * c]; P[1] = newpa[3 * c + 1]; P[2] = newpa[3 * c + 2];
        }
    }
}

/* ------------------------------------------------------ multiple scattering */
/* Library entry of one path (mslibrary.py:433-434): absorber species block,
 * class offset, slot species with slot 0 fastest. Species of sites a and b
 * are overridden by (nsa, nsb) when a >= 0 (the proposed state). */
static inline int orc_ms_entry(const int *S, int ab, int cl, const int *sl,
                               const int *cls_off, int nsp, int nblk,
                               int a, int b, int nsa, int nsb)
{
    int s_ab = S[ab];
    if (a >= 0) s_ab = (ab == a) ? nsa : ((ab == b) ? nsb : s_ab);
    int e = s_ab * nblk + cls_off[cl];
    int pw = 1;
    for (int q = 0; q < 3; ++q) {
        int site = sl[q];
        if (site >= 0) {
            int s = S[site];
            if (a >= 0) s = (site == a) ? nsa : ((site == b) ? nsb : s);
            e += s * pw;
        }
        pw *= nsp;
    }
    return e;
}

void orc_ms_counts(const int *species, int nrep, int natoms,
                   const int *p_abs, const int *p_cls, const int *p_slot, long npath,
                   const int *cls_off, int nsp, int nblk, double *out)
{
    int nent = nsp * nblk;
    for (int c = 0; c < nrep; ++c) {
        const int *S = species + (long)c * natoms;
        double *o = out + (long)c * nent;
        memset(o, 0, sizeof(double) * nent);
        for (long p = 0; p < npath; ++p)
            o[orc_ms_entry(S, p_abs[p], p_cls[p], p_slot + 3 * p, cls_off, nsp, nblk,
                           -1, -1, 0, 0)] += 1.0;
    }
}

/* inc (natoms, M): path ids incident on each site, padded with npath (a
 * dummy path of weight 0), mslibrary.py:383-395. */
void orc_ms_delta(const int *species, int nrep, int natoms,
                  const int *inc, int M, const int *p_abs, const int *p_cls,
                  const int *p_slot, long npath, const int *cls_off, int nsp, int nblk,
                  const int *a, const int *b, const int *nsa, const int *nsb,
                  double *dC)
{
    int nent = nsp * nblk;
    for (int c = 0; c < nrep; ++c) {
        const int *S = species + (long)c * natoms;
        double *o = dC + (long)c * nent;
        memset(o, 0, sizeof(double) * nent);
        for (int half = 0; half < 2; ++half) {
            int site = half ? b[c] : a[c];
            for (int m = 0; m < M; ++m) {
                long pid = inc[(long)site * M + m];
                if (pid >= npath) continue;
                const int *sl = p_slot + 3 * pid;
                if (half) {
                    int has_a = (p_abs[pid] == a[c]) || sl[0] == a[c] || sl[1] == a[c]
                                || sl[2] == a[c];
                    if (has_a) continue;
                }
                int e_old = orc_ms_entry(S, p_abs[pid], p_cls[pid], sl, cls_off, nsp, nblk,
                                         -1, -1, 0, 0);
                int e_new = orc_ms_entry(S, p_abs[pid], p_cls[pid], sl, cls_off, nsp, nblk,
                                         a[c], b[c], nsa[c], nsb[c]);
                o[e_new] += 1.0;
                o[e_old] -= 1.0;
            }
        }
    }
}

/* ---------------------------------------------------------- k -> R transform */
/* chi (rows, nk) on the model grid -> complex chi(R) on the listed bins.
 * idx/frac/inside/w are the reference transform's precomputed arrays
 * (fourier.py:53-67), all length nfft; out_re/out_im (rows, nbins). */
void orc_ft_window(const double *chi, int rows, int nk, const int *idx,
                   const double *frac, const double *inside, const double *w,
                   int nfft, double norm, const int *bins, int nbins,
                   double *out_re, double *out_im)
{
    double *cu = (double *)malloc(sizeof(double) * nfft);
    for (int rw = 0; rw < rows; ++rw) {
        const double *x = chi + (long)rw * nk;
        for (int n = 0; n < nfft; ++n) {
            double a = x[idx[n]], bb = x[idx[n] + 1];
            cu[n] = (a + (bb - a) * frac[n]) * inside[n] * w[n];
        }
        for (int q = 0; q < nbins; ++q) {
            long m = bins[q];
            double sr = 0.0, si = 0.0;
            for (int n = 0; n < nfft; ++n) {
                if (cu[n] == 0.0) continue;
                long j = ((long)n * m) % nfft;
                double ang = ORC_TWO_PI * (double)j / (double)nfft;
                sr += cu[n] * cos(ang);
                si -= cu[n] * sin(ang);
            }
            out_re[(long)rw * nbins + q] = sr * norm;
            out_im[(long)rw * nbins + q] = si * norm;
        }
    }
    free(cu);
}

/* Reduced chi^2 per replica (method_a_rmc.py:211-227) from the window of the
 * model's chi(R): m (nrep, nchan, nwin) complex (im ignored when !cplx, m_re
 * then holds |chi(R)|), target tm, per-component sigma sm (nchan, nwin). */
void orc_chi2(const double *m_re, const double *m_im, int nrep, int nchan, int nwin,
              const double *tm_re, const double *tm_im, const double *sm,
              int nsp, int cplx, int profile, double nfit, double *out)
{
    int nkw = nchan / nsp;
    double *num = (double *)malloc(sizeof(double) * nchan);
    double *den = (double *)malloc(sizeof(double) * nchan);
    for (int c = 0; c < nrep; ++c) {
        const double *mr = m_re + (long)c * nchan * nwin;
        const double *mi = cplx ? m_im + (long)c * nchan * nwin : NULL;
        for (int ch = 0; ch < nchan; ++ch) {
            double nu = 0.0, de = 0.0;
            for (int w = 0; w < nwin; ++w) {
                long o = (long)ch * nwin + w;
                if (cplx) {
                    nu += mr[o] * tm_re[o] + mi[o] * tm_im[o];
                    de += mr[o] * mr[o] + mi[o] * mi[o];
                } else {
                    nu += mr[o] * tm_re[o];
                    de += mr[o] * mr[o];
                }
            }
            num[ch] = nu; den[ch] = de;
        }
        double tot = 0.0;
        for (int ch = 0; ch < nchan; ++ch) {
            double s = 1.0;
            if (profile) {
                int e = ch / nkw;
                double nu = 0.0, de = 0.0;
                for (int q = 0; q < nkw; ++q) { nu += num[e * nkw + q]; de += den[e * nkw + q]; }
                s = nu / fmax(de, 1e-30);
            }
            for (int w = 0; w < nwin; ++w) {
                long o = (long)ch * nwin + w;
                double dr = (mr[o] * s - tm_re[o]) / sm[o];
                double sq = dr * dr;
                if (cplx) {
                    double di = (mi[o] * s - tm_im[o]) / sm[o];
                    sq += di * di;
                }
                tot += sq;
            }
        }
        out[c] = tot / nfit;
    }
    free(num); free(den);
}
