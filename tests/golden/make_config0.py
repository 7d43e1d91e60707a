"""The FP64 reference run of the plain-method configuration, by the oracle on
the CPU (no reference checkout or GPU needed):

    python tests/golden/make_config0.py        # ~7 minutes on one core

Structure: fcc Fe50Ni50, 5x5x5 conventional cells (500 atoms), a0 3.59 A,
species ordered by the seeded nearest-neighbour swap Metropolis run stopped at
alpha1 = -0.08; Fe and Ni K edges; k 2-14 A^-1 at 0.05 (241 points); single
scattering to 5.0 A and exact 3-/4-leg multiple scattering to 5.5 A; the
seeded smooth tables; sigma^2 0.006, S0^2 0.85; target = the model of that
configuration plus N(0, 5e-4) noise (sample position 0); Kaiser window dk 1,
k^1/k^2/k^3, complex chi(R) fitted on 1.4-5.0 A. Sampler: PT-RMC with 8
replicas at geometric temperatures 1e-4 to 1e-1 and 20,000 swap attempts from
a random start (seed 0, swap fraction 1, the reference's displacement
fallback), replica exchange every 25 steps, posterior samples every 50 steps
after 60 % of the run from the 4 rungs whose beta is nearest 0.5
(methods/method_a_rmc.py:401-455, 458-491; chimera/fitrun.py:307-333).

The oracle (oracle/sampler.py) restates the reference's sampler and is pinned
to the reference's own traces (tests/test_oracle_trace.py); its run here is
the FP64 truth the device FP64 sampler is checked against
(tests/test_gpu_config0.py). Saved to tests/golden/config0.npz: the target,
the start configuration, the accept counts per rung, the final and best
states, the best chi^2, the best state's R-factor and first-shell
Warren-Cowley vector, and the posterior Warren-Cowley mean, sd and count.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from chimera_b200 import configs                    # noqa: E402
from chimera_b200 import lattice as L               # noqa: E402
from oracle import sampler as OS                    # noqa: E402

NSTEPS, NREP, EXCH, SEED = 20000, 8, 25, 0
COLLECT_AFTER, COLLECT_EVERY, COLLECT_BETA, NCOLLECT = int(0.6 * NSTEPS), 50, 0.5, 4


def problem():
    prob = configs.Problem(ncell=(5, 5, 5), rmax=5.0, ms=True)
    P = prob.paths
    chans = [OS.Channel(f._idx, f._frac, f._inside, f._w, f.nfft, f._norm,
                        int(prob.ft.chan_edge[c])) for c, f in enumerate(prob.ft.fts)]
    msd = dict(p_abs=P.p_abs, p_cls=P.p_cls, p_slot=P.p_slot, inc=P.inc, cls_off=P.cls_off,
               nblk=P.nblk, T=prob.ms_table)
    nchan = len(chans)
    pr = OS.Problem(prob.cell.ideal, prob.top.i, prob.top.j, prob.top.shift, prob.top.shell,
                    prob.top.sigma2, prob.k, prob.tables.f, prob.tables.delta, prob.tables.lam,
                    prob.tables.s02, chans, np.zeros((nchan, 1024), complex), prob.mask,
                    prob.sigma_R(), prob.nsp, ms=msd)
    sp = prob.target_species[None]
    chi, _, _ = pr.chi_full(prob.cell.ideal[None], sp)
    chi = chi + pr.ms_chi(pr.ms_counts(sp))
    cnt = np.bincount(prob.target_species, minlength=prob.nsp).astype(float)
    chi = chi[0] / np.maximum(cnt, 1)[:, None] + prob.noise_k(0)
    target = pr.observe(chi[None])[0]
    pr.target, pr.tm = target, np.ascontiguousarray(target[:, prob.mask])
    return prob, pr, target


def r_factor(pr, prob, sp, pos):
    """R-factor of one state (chimera/model.py:535-540, profiled per edge)."""
    chi, _, _ = pr.chi_full(pos[None], sp[None])
    chi = chi + pr.ms_chi(pr.ms_counts(sp[None]))
    cnt = np.bincount(sp, minlength=prob.nsp).astype(float)
    m = pr.observe(chi / np.maximum(cnt, 1)[None, :, None])[0][:, prob.mask]
    d = pr.target[:, prob.mask]
    edge = prob.ft.chan_edge
    ne = int(edge.max()) + 1
    num = np.real((np.conj(m) * d).sum(1))
    den = np.real((np.conj(m) * m).sum(1))
    sc = (np.bincount(edge, num, ne) / np.maximum(np.bincount(edge, den, ne), 1e-30))[edge]
    return float((np.abs(m * sc[:, None] - d) ** 2).sum() / (np.abs(d) ** 2).sum())


def wc(prob, sp):
    a = L.warren_cowley(sp, prob.top.i, prob.top.j, prob.top.shift, prob.cell,
                        float(prob.top.r_shell[0]), nsp=prob.nsp)
    return a[np.triu_indices(prob.nsp)]


def main():
    t0 = time.time()
    prob, pr, target = problem()
    sp0 = prob.random_config(SEED)
    smp = OS.PlainSampler(pr, NREP, 1e-4, 1e-1, SEED, 1.0, 0.012, 0.10)
    smp.init_state(sp0, prob.cell.ideal)
    rungs = np.argsort(np.abs(np.log(smp.beta) - np.log(COLLECT_BETA)))[:NCOLLECT]
    acc = np.zeros(NREP, np.int64)
    post = []
    for it in range(NSTEPS):
        acc += np.asarray(smp.step(), np.int64)
        if (it + 1) % EXCH == 0:
            smp.replica_exchange()
        if it >= COLLECT_AFTER and (it + 1) % COLLECT_EVERY == 0:
            post += [wc(prob, smp.species[r]) for r in rungs]
        if (it + 1) % 2000 == 0:
            print(f"  step {it + 1}: best chi^2 {smp.best_chi2.min():.6f} "
                  f"({time.time() - t0:.0f} s)", flush=True)
    b = int(np.argmin(smp.best_chi2))
    bsp, bpos = smp.best_sp[b].astype(np.int32), smp.best_pos[b]
    post = np.array(post)
    out = dict(target=target, species0=sp0.astype(np.int32), accepts=acc,
               final_species=smp.species.astype(np.int8), best_species=bsp.astype(np.int8),
               best_pos=bpos, best_chi2=np.float64(smp.best_chi2[b]),
               best_rfactor=np.float64(r_factor(pr, prob, bsp, bpos)),
               best_alpha=wc(prob, bsp), post_alpha_mean=post.mean(0),
               post_alpha_sd=post.std(0), post_n=np.int64(len(post)),
               exchange_rate=smp.exch_accepted / np.maximum(smp.exch_attempts, 1),
               nsteps=np.int64(NSTEPS), seed=np.int64(SEED))
    np.savez_compressed(os.path.join(HERE, "config0.npz"), **out)
    print(f"wrote config0.npz in {time.time() - t0:.0f} s: best chi^2 {out['best_chi2']:.6f}, "
          f"R {out['best_rfactor']:.3e}, alpha {np.round(out['post_alpha_mean'], 4)}")


if __name__ == "__main__":
    main()
