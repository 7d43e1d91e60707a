"""Synthetic inputs of the benchmark configurations (no public dataset).

  supercell      fcc Fe-Ni (Fe-Ni-Cr) of ncell^3 conventional cells, a0
  tables         `tables.smooth_tables` on 2-14 A^-1 at 0.05 (241 points)
  paths          single scattering to rmax, exact 3-/4-leg MS to 5.5 A half
                 length with `mspaths.synthetic_table`
  disorder       sigma^2 = 0.006 A^2 for every pair, S0^2 = 0.85
  target order   a seeded swap Metropolis run on a nearest-neighbour pair
                 energy (the procedure of chimera/physics.py:234-284), annealed
                 until the first-shell Warren-Cowley alpha of the chosen pair
                 reaches its target (alpha1(Fe-Ni) = -0.08)
  target data    chi(k) of that configuration plus N(0, noise^2) per k point,
                 seed = sample position; complex chi(R) with a Kaiser window
                 (dk = 1, k = 3-13), k^1, k^2, k^3 together, fit 1.4-5.0 A
  sigma_R        the per-component R-space sd the k-space noise produces
"""
from __future__ import annotations

import numpy as np

from . import lattice as L
from . import mspaths as MP
from .fourier import EdgeTransforms
from .tables import smooth_tables, uniform_k


def order_to_alpha(top, composition, target_alpha, pair=(0, 1), seed=0, max_sweeps=200,
                   beta0=0.25):
    """Swap Metropolis on E = V * (number of first-shell `pair` bonds), V = -1,
    at inverse temperature beta0 raised 15% per sweep, stopped at the first
    accepted move that brings alpha1(pair) to target_alpha or below (ordering
    targets, alpha < 0). Returns int32 species."""
    rng = np.random.default_rng(seed)
    n = top.natoms
    sp = L.random_config(n, composition, seed)
    first = top.shell == 0
    nb = top.j[first].reshape(n, -1)             # first-shell neighbours, i-major
    z1 = nb.shape[1]
    A, B = pair
    nA = int((sp == A).sum())
    cB = (sp == B).sum() / n
    nAB = int(((sp[:, None] == A) & (sp[nb] == B)).sum())

    def alpha(m):
        return 1.0 - (m / (nA * z1)) / cB

    def bonds(site, s, skip):
        other = sp[nb[site]]
        keep = nb[site] != skip
        if s == A:
            return int(((other == B) & keep).sum())
        if s == B:
            return int(((other == A) & keep).sum())
        return 0

    beta = beta0
    for _ in range(max_sweeps):
        if alpha(nAB) <= target_alpha:
            break
        for _ in range(n):
            a, b = rng.integers(0, n, 2)
            sa, sb = sp[a], sp[b]
            if sa == sb:
                continue
            before = bonds(a, sa, b) + bonds(b, sb, a)
            after = bonds(a, sb, b) + bonds(b, sa, a)
            d = after - before                    # change of the A-B bond count
            if -d <= 0 or rng.random() < np.exp(beta * d):
                sp[a], sp[b] = sb, sa
                nAB += d
                if alpha(nAB) <= target_alpha:
                    break
        beta *= 1.15
    return sp.astype(np.int32)


class Position:
    """One sample position: target chi(R) and sigma_R for one ladder."""

    def __init__(self, target, sigma_R, mask):
        self.target, self.sigma_R, self.mask = target, sigma_R, mask


class Problem:
    """A supercell with its tables, MS paths, transforms and target order.

    Host data is built eagerly; the device objects (`fm`, the ForwardModel,
    and `ms`, the SupercellMS) are created on first use, so the host part can
    be used where no GPU is present."""

    def __init__(self, elements=("Fe", "Ni"), composition=(0.5, 0.5), ncell=(10, 10, 10),
                 a0=3.59, rmax=5.0, ms=True, ms_half=5.5, sigma2=0.006, s02=0.85,
                 kweights=(1, 2, 3), kmin=3.0, kmax=13.0, window="kaiser", alpha1=-0.08,
                 alpha_pair=(0, 1), noise=5e-4, rwin=(1.4, 5.0), order_seed=0, lattice="fcc"):
        self.elements, self.composition = tuple(elements), tuple(composition)
        self.nsp = len(self.elements)
        self.cell = L.CrystalSupercell(lattice, ncell, a0)
        self.top = L.Topology(self.cell, rmax, sigma2=sigma2)
        self.k = uniform_k()
        self.tables = smooth_tables(self.k, self.elements, s02=s02)
        self.paths = self.ms_table = None
        if ms:
            cls = MP.enumerate_classes(a0, ms_half, lattice)
            self.paths = MP.SupercellPaths(cls, self.cell.ideal, self.cell.H, a0, self.nsp,
                                           conv=self.cell.cell_matrix)
            self.ms_table = MP.synthetic_table(cls, self.nsp, self.k, self.tables.f,
                                               self.tables.delta, self.tables.lam, sigma2,
                                               float(self.top.r_shell[0]),
                                               MP.length_unit(lattice, a0), s02=s02)
        self.ft = EdgeTransforms.build(self.k, kmin, kmax, kweights, nsp=self.nsp,
                                       window=window)
        self.mask = self.ft.window_mask(*rwin)
        self.noise = noise
        self.target_species = order_to_alpha(self.top, self.composition, alpha1, alpha_pair,
                                             seed=order_seed)
        self._chi_t = None
        self._fm = self._ms = None

    @property
    def fm(self):
        if self._fm is None:
            from .forward import ForwardModel
            self._fm = ForwardModel(self.cell, self.tables, self.top.i, self.top.j,
                                    self.top.shift, sigma2=self.top.sigma2, shell=self.top.shell)
        return self._fm

    @property
    def ms(self):
        if self._ms is None and self.paths is not None:
            self._ms = MP.SupercellMS(self.paths, self.ms_table)
        return self._ms

    def alpha1(self, species):
        return L.warren_cowley(np.asarray(species), self.top.i, self.top.j, self.top.shift,
                               self.cell, float(self.top.r_shell[0]), nsp=self.nsp)

    def target_chi(self):
        """Normalised chi(k) (nsp, nk) of the target configuration, MS included."""
        if self._chi_t is None:
            sp = self.target_species[None]
            chi = self.fm.chi(self.cell.ideal[None], sp, normalise=False)
            if self.ms is not None:
                chi = chi + self.ms.full(sp)
            cnt = np.bincount(self.target_species, minlength=self.nsp).astype(float)
            self._chi_t = chi[0].cpu().numpy() / np.maximum(cnt, 1)[:, None]
        return self._chi_t

    def noise_k(self, p):
        return np.random.default_rng(p).normal(0, self.noise, (self.nsp, self.k.size))

    def sigma_R(self):
        """Per-component R-space sd of white k-space noise through each channel
        (a constant of the problem, computed once)."""
        if getattr(self, "_sigma_R", None) is None:
            sig = [self.noise * np.sqrt(0.5 * (np.abs(f.basis()) ** 2).sum(0))
                   for f in self.ft.fts]
            self._sigma_R = np.maximum(np.array(sig), 1e-12)
        return self._sigma_R

    def position(self, p):
        """Target of sample position p: noise seeded by p."""
        chi = self.target_chi() + self.noise_k(p)
        z = np.array([f.to_R(chi[e]) for f, e in zip(self.ft.fts, self.ft.chan_edge)])
        return Position(z, self.sigma_R(), self.mask)

    def random_config(self, seed):
        return L.random_config(self.cell.natoms, self.composition, seed)
