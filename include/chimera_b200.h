/*
 * chimera_b200.h -- C ABI of libchimera_b200.so, the B200 (sm_100a) EXAFS
 * path-sum and parallel-tempering RMC hot path.
 *
 * Conventions
 *   - Every function is extern "C", returns int: CHX_OK (0) or a negative
 *     CHX_ERR_* code; chx_last_error() returns the message of the last failure
 *     on the calling thread. Nothing aborts or traps.
 *   - Every buffer is caller-allocated device memory (row-major, contiguous,
 *     int32 indices, float64 unless stated). The library allocates nothing on
 *     the hot path; kernels that need scratch take a caller buffer sized by the
 *     matching *_scratch_bytes() query.
 *   - Every launch is asynchronous on the caller's stream (`stream` is a
 *     cudaStream_t passed as void*; NULL is the legacy default stream).
 *   - Device-side faults are never provoked: kernels that detect an
 *     out-of-range index or an exhausted bounded wait set a device error word
 *     (CHX_DEVERR_*) that the caller reads back.
 *
 * Reference interfaces each entry point replaces are cited as file:line in
 * the reference project (dluccioni/CHIMERA).
 */
#ifndef CHIMERA_B200_H
#define CHIMERA_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define CHX_API __attribute__((visibility("default")))
#else
#define CHX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CHX_OK 0
#define CHX_ERR_ARG (-1)          /* bad argument (null pointer, size, nsp)   */
#define CHX_ERR_CUDA (-2)         /* a CUDA runtime call failed               */
#define CHX_ERR_UNSUPPORTED (-3)  /* configuration outside the built kernels  */
#define CHX_ERR_SCRATCH (-4)      /* scratch buffer smaller than required     */

/* bits of the device error word */
#define CHX_DEVERR_INDEX 1        /* an index read from a table was out of range */
#define CHX_DEVERR_MSCOUNT 2      /* an MS count delta left the exact range      */

/* precision of the path sums */
#define CHX_FP64 0                /* FP64 throughout (reproduction mode)        */
#define CHX_FP32C 1               /* FP32 transcendentals, FP64 phase reduction  */
                                  /* and FP64 (compensated) accumulation         */

CHX_API int chx_version(void);
/* sizeof / offsetof of the ABI structs, for binding self-checks:
 * 0 sizeof(chx_pairs_t), 1 sizeof(chx_ladder_t),
 * 2 offsetof(chx_ladder_t, exch_acc), 3 offsetof(chx_ladder_t, seed),
 * 4 sizeof(chx_mlp_t), 5 offsetof(chx_ladder_t, log_cap) */
CHX_API int64_t chx_struct_size(int which);
CHX_API int chx_last_error(char *buf, int n);

/* ------------------------------------------------------------------------
 * 1. Entry points of the reference kernel module, same arguments and meaning.
 *    These are what exafs_gpu/kernels.py:get(name, nsp) hands out
 *    (kernels.py:685-686); nsp replaces the -DNSP=<n> compile option
 *    (kernels.py:666-682).
 * ------------------------------------------------------------------------ */

/* exafs_gpu/kernels.py:53-78 (launched forward.py:154) */
CHX_API int chx_compute_r(const double *pos, const int *iidx, const int *jidx,
                  const double *shift, double *r, double *evec,
                  int npairs, int natoms, int nconf, void *stream);

/* exafs_gpu/kernels.py:81-96 (launched forward.py:163) */
CHX_API int chx_build_ptype(const int *species, const int *iidx, const int *jidx, int *ptype,
                    int npairs, int natoms, int nconf, int nsp, void *stream);

/* exafs_gpu/kernels.py:99-163 (launched forward.py:177): full single-scattering
 * path sum, FP64, chi (nconf, nsp, nk) unnormalised. */
CHX_API int chx_chi_forward(const double *r, const int *ptype, const int *shell,
                    const double *sig2, const double *ftab, const double *dtab,
                    const double *lamtab, const double *ktab, const double *drtab,
                    const double *c3tab, const double *s2tab, double *chi,
                    int npairs, int nk, int nconf, double s02, int nsp, void *stream);

/* exafs_gpu/kernels.py:243-325 (launched method_a_rmc.py:267) */
CHX_API int chx_chi_delta(const double *r_old, const int *pt_old, const int *shell,
                  const int *aff, const double *r_new, const int *pt_new,
                  const double *sig2, const double *ftab, const double *dtab,
                  const double *lamtab, const double *ktab, const double *drtab,
                  const double *c3tab, const double *s2tab, double *dchi,
                  int npairs, int nk, int nrep, int maxaff, double s02, int nsp,
                  void *stream);

/* exafs_gpu/kernels.py:328-346 (launched method_a_rmc.py:290) */
CHX_API int chx_commit_move(const int *aff, const double *r_new, const int *pt_new,
                    const uint8_t *accept, double *r_old, int *pt_old,
                    int npairs, int nrep, int maxaff, void *stream);

/* exafs_gpu/kernels.py:362-423 (launched method_a_rmc.py:253); the splitmix64
 * stream keyed (seed, stepc, replica) is reproduced bit for bit. */
CHX_API int chx_propose_select(const int *species, const double *pos, const double *ideal,
                       int *a_out, int *b_out, int *newsa, int *newsb, double *newpa,
                       uint8_t *isswap, int natoms, int nrep, uint64_t seed,
                       uint64_t stepc, double swap_frac, double disp_sigma,
                       double max_disp, void *stream);

/* exafs_gpu/kernels.py:425-488 (launched method_a_rmc.py:260) */
CHX_API int chx_propose_build(const int *species, const double *pos, const int *nbr,
                      const int *rev, const int *iidx, const int *jidx,
                      const double *shift, const int *a_in, const int *b_in,
                      const int *newsa, const int *newsb, const double *newpa,
                      int *aff, double *r_new, int *pt_new, int natoms, int ncoord,
                      int npairs, int nrep, int maxaff, int nsp, void *stream);

/* exafs_gpu/kernels.py:490-511 (launched method_a_rmc.py:294) */
CHX_API int chx_commit_state(const uint8_t *accept, const int *a_in, const int *b_in,
                     const int *newsa, const int *newsb, const double *newpa,
                     const uint8_t *isswap, int *species, double *pos,
                     int natoms, int nrep, void *stream);

/* ------------------------------------------------------------------------
 * 2. Full path sum from positions and species (A1): what ForwardModel.chi
 *    computes with compute_r + build_ptype + chi_forward
 *    (exafs_gpu/forward.py:169-188), without the (nconf, npairs) r/ptype
 *    intermediates. Pair records are built per chunk of pairs into scratch and
 *    staged into shared memory by bulk-async (TMA) copies; each chunk's partial
 *    spectrum is reduced in a fixed order, so the result is deterministic.
 * ------------------------------------------------------------------------ */
typedef struct {
    int natoms, ncoord, npairs, nsp, nk, nshell;
    const int *iidx, *jidx;          /* (npairs), pair p = (iidx[p], jidx[p])   */
    const double *shift;             /* (npairs, 3) periodic image of j         */
    const int *shell;                /* (npairs)                                 */
    const double *sig2;              /* (npairs)                                 */
    const double *ftab;              /* (nsp, nk)   amplitude by scatterer       */
    const double *dtab;              /* (nsp*nsp, nk) phase by pair type         */
    const double *lamtab, *ktab;     /* (nk)                                     */
    const double *drtab;             /* (nshell*nsp*nsp) bond-length offset      */
    const double *c3tab;             /* (nshell) third cumulant                  */
    const double *s2tab;             /* (nshell*nsp*nsp) extra sigma^2           */
    double s02;
} chx_pairs_t;

CHX_API int64_t chx_chi_full_scratch_bytes(const chx_pairs_t *P, int nconf);
/* chi (nconf, nsp, nk) unnormalised; precision CHX_FP64 or CHX_FP32C.
 * Device errors (an index, species or shell out of range; a bulk-copy wait
 * that ran out) set the int32 error word at byte offset
 * chx_chi_full_scratch_bytes(P, nconf) - 256 of the scratch, and make every
 * chi value of the call NaN. */
CHX_API int chx_chi_full(const chx_pairs_t *P, const double *pos, const int *species, int nconf,
                 int precision, double *chi, void *scratch, int64_t scratch_bytes,
                 void *stream);

/* The same path sum for callers that cannot allocate device memory (a host
 * that reaches this library through a foreign-function interface with no
 * device allocator of its own, or code running where allocating is not
 * allowed). No counterpart in the reference: it exists only in this library.
 * The scratch lives in a fixed device array of chx_chi_full_noalloc_max_bytes()
 * bytes (32 MiB) that the library reserves on every GPU that loads it until
 * the process exits; the call allocates nothing. Requests needing more
 * scratch than that are rejected with CHX_ERR_SCRATCH. The first call on a
 * device looks up the array's device address (and may load the module), so
 * make it before any stream capture. The address is kept per device for the
 * life of the process, so calls must not span a reset of that device. All
 * calls on a device share the array: calls that overlap on the GPU race and
 * must be serialised by the caller. The error word lives in the shared array,
 * out of the caller's reach; a device error shows as NaN in every chi value
 * of the call (as for chx_chi_full). */
CHX_API int64_t chx_chi_full_noalloc_max_bytes(void);
CHX_API int chx_chi_full_noalloc(const chx_pairs_t *P, const double *pos, const int *species,
                                 int nconf, int precision, double *chi, void *stream);

/* ------------------------------------------------------------------------
 * 3. Exact supercell multiple scattering (A2): entry counts of every
 *    configuration (chimera/mslibrary.py:436-451) and chi_MS = counts @ table
 *    per absorber block (mslibrary.py:453-457).
 *    A path record is 4 int32: {absorber | entry_offset << 20, slot0, slot1,
 *    slot2}, slots -1 when unused, entry_offset the first library entry of
 *    the path's class (mslibrary.py:275); the path's entry is then
 *    s_abs*nblk + entry_offset + sum_q s_q nsp^q (mslibrary.py:190-198, 433-434).
 * ------------------------------------------------------------------------ */
CHX_API int chx_ms_counts(const int *species, int nconf, int natoms, const int *paths,
                          int64_t npath, int nsp, int nblk, int *counts, void *stream);
/* Entry-count change of each replica's proposal (swap a <-> b to species nsa,
 * nsb; a == b for a displacement, which changes nothing): paths through a and
 * through b, a path through both counted once (mslibrary.py:466-486).
 * inc (natoms, M, 4) holds the records of the paths incident on each site
 * (padding rows -1); dC (nrep, nsp*nblk). */
CHX_API int chx_ms_delta(const int *species, int nrep, int natoms, const int *inc, int M,
                         int nsp, int nblk, const int *a, const int *b, const int *nsa,
                         const int *nsb, int *dC, void *stream);
/* chi (nconf, nsp, nk) += counts (nconf, nsp*nblk) @ T (nsp*nblk, nk), per block */
CHX_API int chx_ms_chi_of(const int *counts, const double *T, int nconf, int nsp, int nblk,
                  int nk, double *chi, void *stream);

/* Pair-type counts over a subset of pairs (e.g. the first shell), one row per
 * configuration: counts (nconf, nsp*nsp), counts[c][a*nsp+b] = number of
 * pairs q with species[c][pi[q]] = a and species[c][pj[q]] = b. The
 * Warren-Cowley parameters of exafs_gpu/lattice.py:167-185 follow as
 * alpha_AB = 1 - (n_AB / n_A) / c_B; the posterior samples of
 * method_a_rmc.py:477-491 (posterior_wc) are taken from them on the device.
 * Out-of-range indices or species set CHX_DEVERR_INDEX in *d_err. */
CHX_API int chx_pair_counts(const int *species, int nconf, int natoms, const int *pi,
                            const int *pj, int npair, int nsp, int *counts, int *d_err,
                            void *stream);

/* ------------------------------------------------------------------------
 * 4. The fused PT-RMC step (A3-A7) and replica exchange (A8) of
 *    methods/method_a_rmc.py:RMCSampler, for a batch of independent ladders.
 *    One CTA per replica slot does: propose (kernels.py:362-423) -> affected
 *    pairs (kernels.py:425-488) -> delta-chi of the pairs (kernels.py:243-325)
 *    and of the MS paths through the two sites (mslibrary.py:466-486) ->
 *    trial chi(R) on the fit window (fourier.py:75-80, multift.py:58-63) ->
 *    profiled chi^2 (method_a_rmc.py:190-227) -> Metropolis
 *    (method_a_rmc.py:280-285) -> commit (kernels.py:328-346, 490-511,
 *    mslibrary.py:488-489) -> best-state retention (method_a_rmc.py:304-307).
 *    Temperatures are exchanged by permuting the rung<->slot maps; the state
 *    never moves, and every rung keeps its own proposal and acceptance
 *    streams (keyed by rung), exactly as when the reference moves the state.
 * ------------------------------------------------------------------------ */
/* The swap surrogate (A11, no reference counterpart): a BF16 MLP with FP32
 * accumulation, 3 hidden ReLU layers of H units, one linear output.
 * Input of a swap of sites lo < hi with species p = S[lo] != q = S[hi]:
 * one-hot row 0..npt-1 the unordered species pair {p, q} (npt =
 * nsp(nsp-1)/2), then for k < 2D (the D neighbours of lo, then of hi, in the
 * feature order) the row npt + k (nsp + 1) + code, code the neighbour's
 * species or nsp where the neighbour is lo or hi; then, when nchain > 0, the
 * row npt + 2D (nsp + 1) + chain of the chain the move belongs to (chain =
 * slot0 + rung in the sampler: ladder and temperature, constant within a
 * step, so a move and its reverse still share the input); plus the scalar
 * feature (ln beta - feat_shift) * feat_scale on row nin. Prediction
 * d^ = sigma * out_scale * net, sigma = +1 if p < q else -1: a swap and its
 * reverse have the same input and opposite predictions, which keeps the
 * two-stage acceptance exact.
 * Parameters live in one FP32 buffer (the masters) and a BF16 copy with the
 * same layout: W1 (nin+1, H) | b1 (H) | W2 (H, H) | b2 | W3 (H, H) | b3 |
 * w4 (H) | b4 (1); row-major [in][out]; compute reads BF16 weights and FP32
 * biases. */
typedef struct chx_mlp {
    int nsp, D, H, nin;              /* nin = npt + 2 D (nsp + 1) + nchain      */
    const uint16_t *W1, *W2, *W3, *w4;   /* BF16 bit patterns */
    const float *b1, *b2, *b3, *b4;
    float out_scale, feat_shift, feat_scale;
    int nchain;                      /* chain rows (0: no chain input)          */
} chx_mlp_t;

/* Parameter count of the layout above. */
CHX_API int64_t chx_mlp_nparam(int nsp, int D, int nchain, int H);
/* Fill the descriptor's pointers for a parameter buffer theta (FP32) and its
 * BF16 copy theta16 (device pointers, same layout). */
CHX_API int chx_mlp_bind(chx_mlp_t *P, int nsp, int D, int nchain, int H, const float *theta,
                         const uint16_t *theta16);
/* Surrogate output for B samples, the same code the sampler step runs:
 * codes (B, 1 + 2D) as above (code[0] the pair row), lnbeta (B), chain (B)
 * (NULL: no chain row); out (B) the network output net (before sigma and
 * out_scale). P is a device pointer. */
CHX_API int chx_mlp_predict(const chx_mlp_t *P, const uint8_t *codes, const float *lnbeta,
                            const int *chain, int B, float *out, void *stream);
/* Training forward (tcgen05 GEMMs over the batch), loss and gradient:
 * loss = mean (net - target)^2; grad (nparam, FP32) overwritten; y (B) the
 * batch outputs; chain (B) sorted ascending (the chain rows' gradient is
 * summed per run of equal chains, in order), or NULL; work:
 * chx_mlp_work_bytes(B, H), which includes the split-K partials of the
 * weight gradients (summed in a fixed order: the gradient is the same on
 * every run). P is a HOST descriptor. */
CHX_API int64_t chx_mlp_work_bytes(int B, int H);
CHX_API int chx_mlp_grad(const chx_mlp_t *P, const uint8_t *codes, const float *lnbeta,
                         const int *chain, const float *target, int B, float *y, float *grad,
                         float *loss, void *work, void *stream);
/* One Adam step (bias-corrected, step number t >= 1) on the FP32 masters,
 * then the BF16 copy: theta -= lr * mhat / (sqrt(vhat) + eps). */
CHX_API int chx_mlp_adam(float *theta, uint16_t *theta16, const float *grad, float *m, float *v,
                         int64_t n, float lr, float beta1, float beta2, float eps, int t,
                         void *stream);

typedef struct {
    /* topology and tables of this ladder's supercell */
    int natoms, ncoord, npairs, nshell, nsp, nk;
    const int *iidx, *jidx, *rev;    /* (npairs), i-major with uniform ncoord    */
    const double *shift;             /* (npairs, 3)                              */
    const int *shell;                /* (npairs)                                 */
    const double *sig2;              /* (npairs)                                 */
    const uint8_t *pair_tab;         /* (npairs) 1: pair may use the shell table */
    const double *ideal;             /* (natoms, 3)                              */
    const double *ftab, *dtab, *lamtab, *ktab, *drtab, *c3tab, *s2tab;
    double s02;
    const double *sstab;             /* (nshell*nsp*nsp, nk) ideal-shell terms, or NULL */
    const float *sstab32;            /* the same table in FP32 (CHX_FP32C), or NULL;
                                        row stride nk rounded up to a multiple of
                                        4, pad columns zero, rows 16-byte aligned
                                        (k points are read four at a time)         */
    /* exact multiple scattering, ms_nblk == 0 when off. The paths through a
       site are ms_M shared templates {class entry offset, 4 position bytes:
       neighbourhood index of the absorber and slots 0-2, 0xFE the site itself,
       0xFF unused} resolved through the site's row of ms_nbr */
    int ms_nblk, ms_M, ms_D;
    const int *ms_tpl;               /* (ms_M, 2) path templates                  */
    const int *ms_nbr;               /* (natoms, ms_D) neighbourhood site indices */
    const double *ms_T;              /* (nsp*ms_nblk, nk)                         */
    const float *ms_T32;             /* the same table in FP32 (CHX_FP32C), or NULL;
                                        row stride and alignment as sstab32        */
    /* pair-interaction prior, etab NULL when off (method_a_rmc.py:147-157,310-320) */
    const double *etab;              /* (nshell*nsp*nsp) eV per directed pair     */
    double energy_beta;
    /* transform (one channel per (edge, k weight), edge-major) and target */
    int nchan, nkw, nwin, nfft, ncoef;
    const int *ft_n0;                /* (nchan) first uniform-grid index, one value
                                        for every channel (coefficients share taps) */
    const int *ft_idx;               /* (nchan, ncoef) resample index             */
    const double *ft_frac;           /* (nchan, ncoef) resample fraction          */
    const double *ft_w;              /* (nchan, ncoef) inside * window * k^w      */
    const int *win_bin;              /* (nwin) R bins of the fit window           */
    const double *chi_extra;         /* (nsp, nk) added before the transform, or NULL */
    double ft_norm;
    const double *tm_re, *tm_im, *sm;/* (nchan, nwin) target window and sigma     */
    const double *w2;                /* (nchan, nwin) 1 / sigma^2                  */
    const double *tnorm;             /* (nchan) sum |target|^2 / sigma^2           */
    int cplx, profile;
    double nfit;
    /* sampler constants */
    uint64_t seed;
    double swap_frac, disp_sigma, max_disp;
    int nrep;                        /* rungs in this ladder                      */
    int slot0;                       /* first slot of this ladder                 */
    const double *beta_rung;         /* (nrep) inverse temperature of each rung   */
    const double *u_stream;          /* (u_steps, nrep) acceptance uniforms, or NULL */
    int64_t u_steps;
    /* state, indexed by slot - slot0 */
    int *species;                    /* (nrep, natoms)                            */
    double *pos;                     /* (nrep, natoms, 3)                         */
    uint8_t *moved;                  /* (nrep, natoms) 1 once displaced           */
    double *chi;                     /* (nrep, nsp, nk) unnormalised, FP64        */
    double *chi2;                    /* (nrep)                                    */
    const double *count;             /* (nrep, nsp) absorber counts               */
    int *rung_of;                    /* (nrep) slot -> rung                       */
    int *slot_of;                    /* (nrep) rung -> slot                       */
    double *best_chi2;               /* (nrep)                                    */
    int *best_sp;                    /* (nrep, natoms)                            */
    double *best_pos;                /* (nrep, natoms, 3)                         */
    int *ms_C;                       /* (nrep, nsp*ms_nblk) entry counts          */
    uint8_t *acc_rung;               /* (nrep) accept flag of the last step, by rung */
    uint8_t *acc_log;                /* (steps, nrep) accept flags of every step of a
                                        launch, by rung, or NULL                     */
    int *n_acc;                      /* (nrep) accepted moves per slot            */
    int *exch_att, *exch_acc;        /* (nrep) exchange bookkeeping per rung pair */
    /* delayed acceptance (no reference counterpart; mlp NULL when off): a
       surrogate predicts each swap's chi^2 change d^ from the species around
       the two sites; stage 1 accepts with min(1, exp(-beta nfit d^ - E)),
       E the exact prior change, and only a move that passes is evaluated
       exactly and accepted with min(1, exp(-beta nfit (d - d^))). */
    const struct chx_mlp *mlp;       /* device descriptor of the surrogate, or NULL */
    const int *feat_nbr;             /* (natoms, feat_D) neighbours of each site in
                                        one translation-invariant order            */
    int feat_D;
    const int *da_on;                /* (1) device word: 1 screens, 0 plain steps  */
    double *da_stat;                 /* (nrep, 4) per slot: moves screened, moves
                                        passed to the exact stage, moves accepted
                                        there, sum of the stage-2 acceptance
                                        probability min(1, exp(-beta nfit (d - d^))) */
    /* swap log for training the surrogate, log_cap 0 when off: every swap
       evaluated exactly writes its features and sigma*d at entry
       ((step - 1) * nrep + slot) mod log_cap */
    uint8_t *log_codes;              /* (log_cap, 1 + 2 feat_D)                  */
    float *log_y;                    /* (log_cap, 4): sigma * d, ln beta, chain
                                        (slot0 + rung), step                     */
    int64_t log_cap;
    /* (nrep) 1 where pos may differ from best_pos (a displacement since
       best_pos was written), 0 where they are equal; NULL: always copy */
    uint8_t *best_stale;
    /* CHX_FP32C, optional: each slot's chi(R) on the fit window in FP64,
       (nrep, nchan, nwin) complex as (re, im) pairs, written in FP64 by
       chx_eval_chi2 (and so by re-anchoring) and kept by the step: a move's
       change alone goes through the FP32 transform and is added to it, so the
       transform's rounding scales with the change, not with chi. NULL: the
       step transforms the whole trial chi in FP32. */
    double *xr;
    /* near ties (with xr and tie_gdiag): x of a Metropolis test is bounded
       against the rounding of the move's change (FP32 terms and MS rows,
       the transform with relative RMS tie_eps per input) at six standard
       deviations; when x - tau and x + tau decide differently, the change is
       recomputed with FP64 terms and rows and both chi^2 with FP64
       transforms, and the test is decided on those;
       tie_stat (nrep, 2): FP64 re-evaluations, decisions they changed. */
    double tie_eps;
    double *tie_stat;
    /* the FP32 terms' share of the near-tie bound (optional, NULL: left out):
       (nsp, nk) the diagonal of G = B W B^H per edge, B the window transform
       of a normalised chi(k) onto the fit bins (all the edge's channels) and
       W = 1 / sigma^2: an independent rounding e(k) of the change adds
       sum_k e(k)^2 G_kk to the expected squared weighted chi(R) norm */
    const double *tie_gdiag;
    /* with xr: (nrep, nsp) the profiled scale of each slot's current state,
       the anchor of the step's one-pass chi^2 (written with xr) */
    double *xs;
    /* with xr, optional: the window transform as split-BF16 tensor-core
       operands, so the step transforms a move's change with three BF16
       products (hi.hi + hi.lo + lo.hi, FP32 accumulation; mma m16n8k16) in
       place of the FP32 DFT. W^T (2 nwin rows: re, im of each window bin;
       ncoef tap columns; the transform norm folded in) in A-fragment order:
       [part hi/lo][m tile (16 rows)][k tile (16 taps)][lane][4 x uint32],
       ft_mt = ceil(2 nwin / 16) m tiles, ft_kt = ceil(ncoef / 16) k tiles,
       zero padded. NULL: the FP32 DFT. */
    const uint32_t *ft_frag;
    int ft_mt, ft_kt;
} chx_ladder_t;

/* Bytes of dynamic shared memory the step kernel needs for these ladders. */
CHX_API int chx_sampler_smem_bytes(const chx_ladder_t *host_ladders, int nladders, int precision);

/* Fill sstab (nshell*nsp*nsp, nk) with the ideal-lattice term of every
 * (shell, pair type) for ladder L: r = shell radius rshell[sh], sigma^2 =
 * s2shell[sh]. FP64. */
CHX_API int chx_shell_table(const chx_ladder_t *L, const double *rshell, const double *s2shell,
                    double *sstab, void *stream);

/* nsteps sampler steps of every slot in one launch (replicas are independent
 * between exchanges, so one CTA runs all steps of its replica). d_ladders:
 * device array of nladders descriptors; slot_ladder (nslots): ladder of each
 * slot. d_stepc: device counter; step s of the launch is step *d_stepc + s + 1
 * (the reference's `_stepc`, first step = 1), and the counter advances by
 * nsteps when the launch completes. (threads, min_blocks): the launch shape,
 * CTA size and CTAs kept resident per SM: (128, 6), (256, 3) or (256, 4);
 * (0, 0) picks (256, 3). d_err: device error word. */
CHX_API int chx_sampler_step(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders,
                             int nladders, const int *slot_ladder, int nslots, int precision,
                             int nsteps, int threads, int min_blocks, uint64_t *d_stepc,
                             int *d_ticket, int *d_err, void *stream);

/* chi^2 of every slot's state chi (chi_in NULL) or of chi_in (nslots, nsp, nk)
 * with absorber counts count_in (nslots, nsp) (count NULL: the state's), by
 * the step's own transform and profiled chi^2, into out (nslots). */
CHX_API int chx_eval_chi2(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders,
                          int nladders, const int *slot_ladder, int nslots, int precision,
                          const double *chi_in, const double *count_in, double *out,
                          void *stream);

/* FP64 re-anchoring (no reference counterpart; the reference accumulates its
 * running chi in FP64 forever, method_a_rmc.py:298): replace the running chi of
 * every slot with mask[slot] != 0 (mask NULL: every slot) by a fresh FP64
 * recompute from its species, positions and MS entry counts, in the
 * pair-count form (pairs on ideal sites counted per (shell, type) and
 * contracted with the FP64 term table sstab; displaced pairs by the FP64 pair
 * term), and reset its accepted-move counter. Uses the counted form where
 * sstab is set; nk <= 512. The work of a slot is spread over the GPU in
 * chunks of 1,024 pairs whose partial spectra are summed in chunk order
 * (deterministic); scratch (caller-owned) is sized by
 * chx_reanchor_scratch_bytes(host_ladders, nladders, max_due) with
 * max_due = nslots for chx_reanchor. */
/* chi^2 of each slot with mask[slot] != 0 (mask NULL: every slot) from its own
 * chi, written to the slot's chi2 (and, in CHX_FP32C with xr, its FP64
 * chi(R)): the refresh after a re-anchoring of those slots
 * (method_a_rmc.py:180 evaluates the start state the same way). */
CHX_API int chx_refresh_chi2(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders,
                             int nladders, const int *slot_ladder, int nslots, int precision,
                             const uint8_t *mask, void *stream);
CHX_API int64_t chx_reanchor_scratch_bytes(const chx_ladder_t *host_ladders, int nladders,
                                           int max_due);
CHX_API int chx_reanchor(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders,
                         int nladders, const int *slot_ladder, int nslots, const uint8_t *mask,
                         void *scratch, int64_t scratch_bytes, int *d_err, void *stream);
/* The same re-anchoring decided on the device, for use inside a captured
 * exchange period: the slots whose accepted-move counter reached `every`
 * (config 1: 1,000), at most max_due of them per call in slot order (the rest
 * wait for the next call), are recomputed in FP64 as above and their chi^2
 * refreshed in `precision`; due[slot] (device, nslots bytes) records which,
 * and the device counter *count (may be NULL) grows by their number.
 * No counterpart in the reference (closest: method_a_rmc.py:436-448). */
CHX_API int chx_reanchor_due(const chx_ladder_t *d_ladders, const chx_ladder_t *host_ladders,
                             int nladders, const int *slot_ladder, int nslots, int every,
                             int max_due, int precision, uint8_t *due, unsigned long long *count,
                             void *scratch, int64_t scratch_bytes, int *d_err, void *stream);

/* Replica exchange decided on the device (method_a_rmc.py:332-373): alternate
 * adjacent rung pairs from a random start parity, accept d >= 0 or
 * u < exp(max(d, -60)) with d = (b_i - b_{i+1})(E_i - E_{i+1}) nfit. The
 * uniforms come from a splitmix64 stream keyed (seed, *round_key), round_key
 * a device word (the step counter), so a captured graph draws fresh uniforms
 * on every replay. */
CHX_API int chx_replica_exchange(const chx_ladder_t *d_ladders, int nladders,
                                 const uint64_t *round_key, void *stream);

/* Apply a host-decided exchange: order (nrep) as the reference builds it
 * (method_a_rmc.py:344-366); rung i takes the state rung order[i] held. */
CHX_API int chx_apply_exchange(const chx_ladder_t *d_ladders, int ladder, const int *order,
                       void *stream);

/* ------------------------------------------------------------------------
 * 5. Windowed FT of a batch of spectra to chi(R) on arbitrary R points (A5,
 *    fourier.py:75-80 generalised to a direct transform). X (rows, nR) complex
 *    interleaved; basis (nk, nR) complex = w(k) k^kw dk/sqrt(pi) e^{-2ikR}.
 *    precision: 0 FP64 (SIMT), 1 FP32 (SIMT), 2 split-BF16 three-product on
 *    the tcgen05 tensor cores with FP32 accumulation, 3 TF32 on the tcgen05
 *    tensor cores (one product, FP32 accumulation). Precisions 2 and 3 write
 *    a device error word (CHX_DEVERR_*) into the first 4 bytes of scratch
 *    (256-byte aligned) and need out 16-byte aligned (it is written by TMA
 *    tensor stores).
 * ------------------------------------------------------------------------ */
CHX_API int chx_ft_batch(const double *chi, int rows, int nk, const double *basis, int nR,
                 int precision, double *out, void *scratch, int64_t scratch_bytes,
                 void *stream);

/* The fused form of the windowed FT for a profiled chi^2 (config 2's form):
 * the same tensor-core contraction (precision 2 split-BF16, 3 TF32) of chi
 * (rows, nk) with basis (nk, 2 nR) as chx_ft_batch, but instead of chi(R) its
 * epilogue writes each row's sums against a target and weights over the bins
 * with w != 0 (the fit window), anchored at a scale s0: sums (rows, 7) =
 * {Re<m,t>, <m,m>, R = sum w |s0 m - t|^2, Q = sum w Re(m (s0 m - t)*),
 * P = sum w |m|^2, Ru = sum |s0 m - t|^2, Qu = sum Re(m (s0 m - t)*)},
 * 56 bytes per row in place of 16 nR. The profiled scale
 * s = sum Re<m,t> / sum <m,m> (over an edge's channels),
 * sum w |s m - t|^2 = R + 2 (s - s0) Q + (s - s0)^2 P and the R-factor
 * numerator Ru + 2 (s - s0) Qu + (s - s0)^2 <m,m> follow on the host
 * (method_a_rmc.py:190-227, model.py:497-540); with s0 near s nothing
 * cancels. Products and the sums within one 128-column tile are FP32 (the
 * accumulator's precision), the sums across tiles FP64. target (nR, 2) re/im, weight (nR) = 1 / sigma^2 in the window, 0
 * outside. Scratch: chx_ft_window_sums_scratch_bytes (256-byte aligned). */
CHX_API int64_t chx_ft_window_sums_scratch_bytes(int rows, int nk, int nR, int precision);
CHX_API int chx_ft_window_sums(const double *chi, int rows, int nk, const double *basis, int nR,
                               const double *target, const double *weight, double s0,
                               int precision, double *sums, void *scratch,
                               int64_t scratch_bytes, void *stream);
CHX_API int64_t chx_ft_batch_scratch_bytes(int rows, int nk, int nR, int precision);

/* ------------------------------------------------------------------------
 * Pair-count (shell) calibration objective, for a population of parameter sets
 *
 * Replaces the host loop over a differential-evolution population of the
 * reference's ShellModel.r_factor (chimera/shellmodel.py:427-440; basis
 * :290-336, chi_k :411-413, chi_ms :338-356 with multiscat.py:133-145,
 * transforms :358-372; called by chimera/calibrate.py:364-371, 473-478).
 * One row of `params` per member, FP64, laid out as
 *   [a0, sigma_scale, ms_amp, ms_c, kmin, kmax, dE0[nsp],
 *    sigma_shell_scale[nshell], dr[nsp*nsp], c3[nshell], c4[nshell],
 *    sigma_pair[nsp*nsp], ms_amp_edge[nsp]]
 * (chx_shell_nparam values). Per member: the basis B[a,b,s](k) at its
 * parameters contracted with the pair counts N, plus the averaged MS term;
 * each channel (edge e, k weight w; edge-major) resampled from the member's
 * k axis sqrt(k^2 - etok dE0[e]) onto n dk, times the Hanning window of its
 * kmin, kmax (taper dk_win) and k^w, and transformed (e^{-2ikR}, dk/sqrt(pi))
 * on the fitted FFT bins; one amplitude per edge profiled out and the
 * R-factor over all channels (model.py:497-545).
 * ------------------------------------------------------------------------ */
typedef struct {
    int nsp, nshell, nk, nkw, nbin, nfft;
    int magnitude;                   /* 1: fit |chi(R)| to real data          */
    double a0_ref, s02, dk_win, dk, etok;
    const double *k;                 /* (nk) model k grid (k_phys)            */
    const double *f, *delta, *lam;   /* (nsp, nk), (nsp*nsp, nk), (nk)        */
    const double *shells_ref;        /* (nshell) shell radii at a0_ref        */
    const double *sigma2_ref;        /* (nshell) reference sigma^2 per shell  */
    const double *shell_mult;        /* (nshell) coordination per shell       */
    const double *N;                 /* (nsp, nsp, nshell) ordered pair counts */
    const int *kweight;              /* (nkw)                                  */
    const int *bins;                 /* (nbin) FFT bins of the fitted points   */
    const double *data;              /* (nsp*nkw, nbin, 2) re, im (im unused
                                        for magnitude data)                   */
    /* averaged multiple scattering, npath == 0 when off */
    int npath;
    double ms_dnn;                   /* nearest-neighbour distance of the paths */
    const int *ms_abs;               /* (npath) absorber species of each path  */
    const double *ms_reff, *ms_deg;  /* (npath)                               */
    const double *ms_F, *ms_D, *ms_L; /* (npath, nk)                          */
    /* Fisher-bound extensions (chimera/shellmodel.py:449-593): per-member
       pair counts (P, nsp, nsp, nshell) in place of N, or NULL; the residual
       (scale m - data) / sigma of every member (P, nchan, nbin, 2: re, im)
       written to resid when not NULL, sigma (nchan, nbin) or NULL for 1;
       profile 0 holds the amplitudes at 1 */
    const double *N_member;
    double *resid;
    const double *sigma;
    int profile;
} chx_shell_t;

CHX_API int chx_shell_nparam(int nsp, int nshell);
/* rf (P), scales (P, nsp) per-edge amplitudes; a member whose k axis or
 * window leaves the built tap range gets rf = NaN. */
CHX_API int chx_shell_rfactor(const chx_shell_t *S, const double *params, int P, double *rf,
                              double *scales, void *stream);

/* ------------------------------------------------------------------------
 * Curved-wave multiple-scattering path trace (K edge, orientation averaged)
 *
 * Replaces the reference's path_trace kernel and its host driver
 * (exafs_gpu/abinitio/pathsum.py:158-343, CPU twin trace_numpy :106-126,
 * called by path_sum / provider.py:173-225): Tr_{l=1} of every path's
 * product G(a_N) t_N D_N ... t_1 D_1 G(a_0) and the closing rotation, one
 * CTA per (energy, path), FP64 complex. Complex values are (re, im) pairs.
 * ------------------------------------------------------------------------ */
typedef struct {
    int npath, maxs, ne, ntype, nlt, glmax;  /* glmax: the tables' lmax (<= 40)  */
    const int *nsc;                  /* (npath) scatterers per path              */
    const int *typ;                  /* (npath, maxs) scatterer types            */
    const double *leg;               /* (npath, maxs+1) leg lengths (bohr)       */
    const double *eul;               /* (npath, maxs+1, 3) zyz Euler angles of the
                                        frame changes, the closing one last      */
    const double *p;                 /* (ne, 2) complex momentum (bohr^-1)       */
    const double *t;                 /* (ntype, ne, nlt, 2) t_l = (S_l - 1)/2     */
    const int *lmax;                 /* (npath, ne) angular momentum cut, <= glmax */
    const int *goff, *gcnt;          /* ((glmax+1)^3) runs of the propagator
                                        coefficients A^m_{l'l l''}, [|m|][l'][l] */
    const int *glpp;                 /* l'' of every run entry                   */
    const double *gA;                /* (nruns, 2) A of every run entry          */
    const int64_t *doff;             /* (glmax+2) offsets of Delta^l = d^l(pi/2) */
    const double *dflat;             /* Delta^l[m''+l][m+l] blocks               */
} chx_path_t;

/* out (npath, ne, 2): the trace of every path at every energy (NaN for a path
 * whose sizes or types are out of range). */
CHX_API int chx_path_trace(const chx_path_t *P, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CHIMERA_B200_H */
