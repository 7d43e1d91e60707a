"""The plain PT-RMC loop on the CPU (test infrastructure: the checker and the
CPU baseline). Restates methods/method_a_rmc.py step by step with NumPy in
place of CuPy:

  init          :166-184   state, full chi (kernels.py:53-163), MS init
  chi2          :190-227   profiled per-edge scale, complex/magnitude target
  step          :250-308   propose_select, propose_build, chi_delta, MS
                           delta, trial chi^2, Metropolis, commits, best
  exchange      :332-373   host PCG64 exchange on adjacent rungs
  run           :401-455   exchange every `exchange_every` steps

The transform is the reference's: resample, window, np.fft of length nfft,
first nfft/2 bins, times dk/sqrt(pi) (exafs_gpu/fourier.py:69-80), one per
(edge, k weight) channel plus chi_extra (chimera/multift.py:58-63).
Random streams: proposals splitmix64 keyed (seed, step, replica) inside the
C kernels; acceptance PCG64(seed).random(nrep) per step; exchange a second
PCG64(seed).
"""
from __future__ import annotations

import numpy as np

from . import kernels as K


class Channel:
    """One channel's transform set-up (fourier.py:39-67 arrays)."""

    def __init__(self, idx, frac, inside, w, nfft, norm, edge):
        self.idx, self.frac, self.inside, self.w = idx, frac, inside, w
        self.nfft, self.norm, self.edge = int(nfft), float(norm), int(edge)

    def to_R(self, chi):
        a = chi[..., self.idx]
        b = chi[..., self.idx + 1]
        cu = (a + (b - a) * self.frac) * self.inside * self.w
        return np.fft.fft(cu, n=self.nfft, axis=-1)[..., : self.nfft // 2] * self.norm


def ft_setup(k_model, kmin, kmax, kweight, dk_win=1.0, nfft=2048, dk=0.05, window=None):
    """The reference transform's set-up arrays (fourier.py:25-67); `window`
    overrides the Hanning window with given values on the uniform grid."""
    k_model = np.asarray(k_model, float)
    ku = np.arange(nfft) * dk
    if window is None:
        w = np.zeros_like(ku)
        w[(ku >= kmin + dk_win / 2) & (ku <= kmax - dk_win / 2)] = 1.0
        lo = (ku > kmin - dk_win / 2) & (ku < kmin + dk_win / 2)
        w[lo] = 0.5 * (1 + np.sin(np.pi * (ku[lo] - kmin) / dk_win))
        hi = (ku > kmax - dk_win / 2) & (ku < kmax + dk_win / 2)
        w[hi] = 0.5 * (1 - np.sin(np.pi * (ku[hi] - kmax) / dk_win))
    else:
        w = np.asarray(window, float).copy()
    w[ku > k_model.max()] = 0.0
    w[ku < k_model.min()] = 0.0
    weight = w * ku ** kweight
    idx = np.clip(np.searchsorted(k_model, ku) - 1, 0, k_model.size - 2)
    span = np.maximum(k_model[idx + 1] - k_model[idx], 1e-12)
    frac = np.clip((ku - k_model[idx]) / span, 0.0, 1.0)
    inside = (ku >= k_model[0]) & (ku <= k_model[-1])
    return dict(idx=idx, frac=frac * inside, inside=inside.astype(np.float64), w=weight,
                nfft=nfft, norm=dk / np.sqrt(np.pi), R=np.arange(nfft // 2) * np.pi / (nfft * dk))


class Problem:
    """Everything the plain sampler needs, as host arrays."""

    def __init__(self, ideal, i, j, shift, shell, sig2, k, f, delta, lam, s02, channels,
                 target, mask, sigR, nsp, dr=None, c3=None, s2tab=None, chi_extra=None,
                 ms=None, etab=None, energy_beta=0.0):
        self.ideal = np.ascontiguousarray(ideal, np.float64)
        self.natoms = self.ideal.shape[0]
        self.i = np.ascontiguousarray(i, np.int32)
        self.j = np.ascontiguousarray(j, np.int32)
        self.shift = np.ascontiguousarray(shift, np.float64)
        self.shell = np.ascontiguousarray(shell, np.int32)
        self.sig2 = np.ascontiguousarray(sig2, np.float64)
        self.npairs = self.i.size
        self.nsp = int(nsp)
        self.nshell = int(self.shell.max()) + 1
        nn = self.nsp * self.nsp
        self.k = np.ascontiguousarray(k, np.float64)
        self.nk = self.k.size
        self.f = np.ascontiguousarray(f, np.float64)
        self.delta = np.ascontiguousarray(np.asarray(delta).reshape(nn, -1), np.float64)
        self.lam = np.ascontiguousarray(lam, np.float64)
        self.s02 = float(s02)
        z = lambda n: np.zeros(n)
        self.dr = np.ascontiguousarray(z(self.nshell * nn) if dr is None else dr, np.float64).ravel()
        self.c3 = np.ascontiguousarray(z(self.nshell) if c3 is None else c3, np.float64).ravel()
        self.s2tab = np.ascontiguousarray(z(self.nshell * nn) if s2tab is None else s2tab,
                                          np.float64).ravel()
        self.channels = channels
        self.nchan = len(channels)
        self.nkw = self.nchan // self.nsp
        self.target = np.asarray(target)
        self.mask = np.asarray(mask, bool)
        self.sigR = np.asarray(sigR, float)
        self.cplx = bool(np.iscomplexobj(self.target))
        self.tm = np.ascontiguousarray(self.target[:, self.mask])
        self.sm = np.ascontiguousarray(self.sigR[:, self.mask])
        self.nfit = int(self.mask.sum()) * self.nchan * (2 if self.cplx else 1)
        self.chi_extra = chi_extra
        self.ms = ms                     # dict(p_abs, p_cls, p_slot, inc, cls_off, nblk, T)
        self.etab = etab
        self.energy_beta = float(energy_beta)
        counts = np.bincount(self.i, minlength=self.natoms)
        self.ncoord = int(counts[0])
        key = self.i.astype(np.int64) * self.natoms + self.j
        rkey = self.j.astype(np.int64) * self.natoms + self.i
        order = np.argsort(key)
        self.rev = order[np.searchsorted(key[order], rkey)].astype(np.int32)
        self.nbr = np.arange(self.npairs, dtype=np.int32).reshape(self.natoms, self.ncoord)

    # ------------------------------------------------------------ physics
    def chi_full(self, pos, species):
        pos = np.ascontiguousarray(pos, np.float64)
        species = np.ascontiguousarray(species, np.int32)
        n = pos.shape[0]
        r = np.zeros((n, self.npairs))
        pt = np.zeros((n, self.npairs), np.int32)
        K.compute_r(pos, self.i, self.j, self.shift, r, None, self.npairs, self.natoms, n)
        K.build_ptype(species, self.i, self.j, pt, self.npairs, self.natoms, n, self.nsp)
        chi = np.zeros((n, self.nsp, self.nk))
        K.chi_forward(r, pt, self.shell, self.sig2, self.f, self.delta, self.lam, self.k,
                      self.dr, self.c3, self.s2tab, chi, self.npairs, self.nk, n, self.s02,
                      self.nsp)
        return chi, r, pt

    def ms_counts(self, species):
        m = self.ms
        return K.ms_counts(species, m["p_abs"], m["p_cls"], m["p_slot"], m["cls_off"],
                           self.nsp, m["nblk"])

    def ms_chi(self, C):
        T, nb = self.ms["T"], self.ms["nblk"]
        return np.stack([C[:, a * nb:(a + 1) * nb] @ T[a * nb:(a + 1) * nb]
                         for a in range(self.nsp)], axis=1)

    def observe(self, chi_norm):
        x = chi_norm if self.chi_extra is None else chi_norm + self.chi_extra
        z = np.stack([c.to_R(x[:, c.edge, :]) for c in self.channels], axis=1)
        return z if self.cplx else np.abs(z)

    def chi2(self, chi_un, count):
        chi = chi_un / np.maximum(count, 1.0)[:, :, None]
        m = self.observe(chi)[:, :, self.mask]
        return K.chi2(m, self.tm, self.sm, self.nsp, self.profile, self.nfit)

    profile = True


class PlainSampler:
    """CPU PT-RMC on one ladder (reference semantics, see module doc)."""

    def __init__(self, prob: Problem, nrep, tmin, tmax, seed, swap_frac, disp_sigma, max_disp,
                 profile_scale=True):
        self.p = prob
        prob.profile = bool(profile_scale)
        self.nrep = int(nrep)
        self.seed = int(seed)
        self.rng = np.random.default_rng(seed)
        self.urng = np.random.default_rng(seed)
        self.swap_frac, self.disp_sigma, self.max_disp = swap_frac, disp_sigma, max_disp
        self.beta = 1.0 / np.geomspace(tmin, tmax, nrep)
        self.maxaff = 4 * prob.ncoord
        self.stepc = 0
        self.exch_attempts = np.zeros(max(nrep - 1, 1))
        self.exch_accepted = np.zeros(max(nrep - 1, 1))

    def init_state(self, species0, pos0):
        p, n = self.p, self.nrep
        self.species = np.ascontiguousarray(np.repeat(species0[None], n, 0), np.int32)
        self.pos = np.ascontiguousarray(np.repeat(pos0[None], n, 0), np.float64)
        self.ideal = np.ascontiguousarray(np.repeat(p.ideal[None], n, 0))
        # every replica starts from the same configuration: evaluate it once
        chi1, r1, pt1 = p.chi_full(self.pos[:1], self.species[:1])
        self.chi = np.repeat(chi1, n, 0)
        self.r = np.ascontiguousarray(np.repeat(r1, n, 0))
        self.ptype = np.ascontiguousarray(np.repeat(pt1, n, 0))
        if p.ms is not None:
            self.C = np.repeat(p.ms_counts(self.species[:1]), n, 0)
            self.chi = self.chi + p.ms_chi(self.C)
        self.count = np.stack([(self.species == s).sum(1) for s in range(p.nsp)],
                              axis=1).astype(np.float64)
        self.chi2 = p.chi2(self.chi, self.count)
        self.best_chi2 = self.chi2.copy()
        self.best_sp = self.species.copy()
        self.best_pos = self.pos.copy()

    def step(self):
        p, n, m = self.p, self.nrep, self.maxaff
        self.stepc += 1
        a = np.zeros(n, np.int32); b = np.zeros(n, np.int32)
        nsa = np.zeros(n, np.int32); nsb = np.zeros(n, np.int32)
        npa = np.zeros((n, 3)); isswap = np.zeros(n, np.uint8)
        K.propose_select(self.species, self.pos, self.ideal, a, b, nsa, nsb, npa, isswap,
                         p.natoms, n, self.seed, self.stepc, self.swap_frac, self.disp_sigma,
                         self.max_disp)
        aff = np.zeros((n, m), np.int32); rnew = np.zeros((n, m)); ptnew = np.zeros((n, m), np.int32)
        K.propose_build(self.species, self.pos, p.nbr, p.rev, p.i, p.j, p.shift, a, b, nsa, nsb,
                        npa, aff, rnew, ptnew, p.natoms, p.ncoord, p.npairs, n, m, p.nsp)
        dchi = np.zeros((n, p.nsp, p.nk))
        K.chi_delta(self.r, self.ptype, p.shell, aff, rnew, ptnew, p.sig2, p.f, p.delta, p.lam,
                    p.k, p.dr, p.c3, p.s2tab, dchi, p.npairs, p.nk, n, m, p.s02, p.nsp)
        dC = None
        if p.ms is not None:
            ms = p.ms
            dC = K.ms_delta(self.species, ms["inc"], ms["p_abs"], ms["p_cls"], ms["p_slot"],
                            ms["p_abs"].size, ms["cls_off"], p.nsp, ms["nblk"], a, b, nsa, nsb)
            dchi = dchi + p.ms_chi(dC)
        trial = self.chi + dchi
        c2 = p.chi2(trial, self.count)
        x = self.beta * (c2 - self.chi2) * p.nfit
        if p.etab is not None:
            nn = p.nsp * p.nsp
            valid = aff >= 0
            affc = np.maximum(aff, 0)
            sh = p.shell[affc]
            pold = np.take_along_axis(self.ptype, affc, axis=1)
            d = p.etab[sh * nn + ptnew] - p.etab[sh * nn + pold]
            x = x + p.energy_beta * (d * valid).sum(axis=1)
        u = self.urng.random(n)
        with np.errstate(over="ignore"):       # exp(-x) for x <= 0 is not used
            acc = (x <= 0) | (u < np.exp(-np.minimum(x, 60.0)))
        # the step's proposals and exact chi^2 changes, by rung (read by tests)
        self.last = dict(a=a.copy(), b=b.copy(), swap=isswap.copy(), species=self.species.copy(),
                         d=c2 - self.chi2)
        accb = acc.astype(np.uint8)
        if dC is not None:
            self.C = self.C + dC * acc[:, None]
        K.commit_move(aff, rnew, ptnew, accb, self.r, self.ptype, p.npairs, n, m)
        K.commit_state(accb, a, b, nsa, nsb, npa, isswap, self.species, self.pos, p.natoms, n)
        self.chi = np.where(acc[:, None, None], trial, self.chi)
        self.chi2 = np.where(acc, c2, self.chi2)
        imp = self.chi2 < self.best_chi2
        self.best_chi2 = np.where(imp, self.chi2, self.best_chi2)
        self.best_sp = np.where(imp[:, None], self.species, self.best_sp)
        self.best_pos = np.where(imp[:, None, None], self.pos, self.best_pos)
        return acc

    def replica_exchange(self):
        c2 = self.chi2
        order = np.arange(self.nrep)
        start = self.rng.integers(0, 2)
        nsw = 0
        for i in range(start, self.nrep - 1, 2):
            d = (self.beta[i] - self.beta[i + 1]) * (c2[order[i]] - c2[order[i + 1]]) * self.p.nfit
            ok = d >= 0 or self.rng.random() < np.exp(max(d, -60.0))
            self.exch_attempts[i] += 1
            if ok:
                order[i], order[i + 1] = order[i + 1], order[i]
                nsw += 1
                self.exch_accepted[i] += 1
        if nsw:
            for name in ("chi", "chi2", "pos", "species", "r", "ptype", "count", "best_chi2",
                         "best_sp", "best_pos"):
                setattr(self, name, np.ascontiguousarray(getattr(self, name)[order]))
            if self.p.ms is not None:
                self.C = self.C[order]
        return order

    def run(self, nsteps, exchange_every=25, trace=None):
        for it in range(nsteps):
            acc = self.step()
            if trace is not None:
                trace.append(acc.copy())
            if exchange_every and (it + 1) % exchange_every == 0:
                self.replica_exchange()
        return self
