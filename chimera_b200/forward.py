"""Device forward model: configuration -> chi(k) (exafs_gpu/forward.py).

`ForwardModel` keeps the reference class's constructor, attributes and
methods (forward.py:50-188): the tables and topology live on the device as
`d_*` tensors that callers may reassign (chimera/model.py:263, 278 assign
`d_shift` and `d_sig2` directly), `set_dr` / `set_sig2_types` / `set_c3`
fill the per-(shell, type) tables, `distances` and `ptypes` run the
reference kernels' equivalents, and `chi` evaluates the full path sum.

`chi(pos, species)` without precomputed r/ptype runs the B200 path sum
(`chx_chi_full`: pair records staged by bulk-async copies, k-vectorised
accumulation, deterministic reduction). With r and ptype given it runs the
reference kernel's equivalent (`chx_chi_forward`). `precision` selects FP64
(default, the reference's arithmetic) or FP32 transcendentals with FP64 phase
reduction and accumulation.
"""
from __future__ import annotations

import numpy as np

from . import _native as N

FP64, FP32C = 0, 1


def thermal_sigma2_uniform(npairs, sigma2):
    """A uniform per-pair sigma^2 (the benchmark configurations' 0.006 A^2)."""
    return np.full(npairs, float(sigma2))


class ForwardModel:
    """Holds device-resident tables and topology; evaluates chi."""

    def __init__(self, cell, tables, i_idx, j_idx, shift, sigma2=None, shell=None):
        import torch
        N.require_cuda()
        self.cell = cell
        self.natoms = cell.natoms
        self.npairs = int(np.asarray(i_idx).size)
        k, f, delta, lam = tables.as_float64()
        self.nk = int(k.size)
        self.nsp = int(f.shape[0])
        self.s02 = float(tables.s02)
        if shell is None:
            shell = np.zeros(self.npairs, np.int32)
        shell = np.ascontiguousarray(shell, np.int32)
        assert shell.shape == (self.npairs,), "shell must be one index per pair"
        self.nshell = int(shell.max()) + 1
        self.shell = shell
        z = np.bincount(np.asarray(i_idx), minlength=self.natoms)
        self.ncoord = int(z[0]) if z.min() == z.max() else 0
        self.d_shell = N.to_dev(shell)
        self.dr = np.zeros((self.nshell, self.nsp, self.nsp))
        self.c3 = np.zeros(self.nshell)
        self.s2types = np.zeros((self.nshell, self.nsp, self.nsp))
        self.d_dr = torch.zeros(self.nshell * self.nsp * self.nsp, dtype=torch.float64, device="cuda")
        self.d_c3 = torch.zeros(self.nshell, dtype=torch.float64, device="cuda")
        self.d_s2tab = torch.zeros_like(self.d_dr)
        self.tables = tables
        self.k = k
        self.d_k = N.to_dev(k)
        self.d_f = N.to_dev(f)
        dflat = np.ascontiguousarray(delta.reshape(self.nsp ** 2, -1))
        self.d_delta = N.to_dev(dflat)
        self.d_cosd = N.to_dev(np.cos(dflat))
        self.d_sind = N.to_dev(np.sin(dflat))
        self.d_lam = N.to_dev(lam)
        self.i_idx = np.ascontiguousarray(i_idx, np.int32)
        self.j_idx = np.ascontiguousarray(j_idx, np.int32)
        self.d_i = N.to_dev(self.i_idx)
        self.d_j = N.to_dev(self.j_idx)
        self.d_shift = N.to_dev(np.ascontiguousarray(shift, np.float64))
        if sigma2 is None:
            sigma2 = np.zeros(self.npairs)
        self.d_sig2 = N.to_dev(np.ascontiguousarray(sigma2, np.float64))

    # ------------------------------------------------------ cumulant physics
    def set_dr(self, dr):
        dr = np.asarray(dr, np.float64)
        full = np.zeros((self.nshell, self.nsp, self.nsp))
        if dr.ndim == 2:
            full[0] = dr
        else:
            assert dr.shape == full.shape, f"dr must be {full.shape} or (nsp, nsp)"
            full[:] = dr
        self.dr = full
        self.d_dr = N.to_dev(full.reshape(-1))
        return self

    def set_sig2_types(self, s2):
        s2 = np.asarray(s2, np.float64)
        full = np.zeros((self.nshell, self.nsp, self.nsp))
        if s2.ndim == 2:
            full[0] = s2
        else:
            n = min(self.nshell, s2.shape[0])
            full[:n] = s2[:n]
        self.s2types = full
        self.d_s2tab = N.to_dev(full.reshape(-1))
        return self

    def set_c3(self, c3):
        c3 = np.atleast_1d(np.asarray(c3, np.float64))
        full = np.zeros(self.nshell)
        if c3.size == 1:
            full[0] = c3[0]
        else:
            assert c3.shape == (self.nshell,), f"c3 must have {self.nshell} entries"
            full[:] = c3
        self.c3 = full
        self.d_c3 = N.to_dev(full)
        return self

    # ---------------------------------------------------------------- helpers
    def pairs_desc(self):
        """chx_pairs_t over the current device tables (kept alive by self)."""
        P = N.Pairs()
        P.natoms, P.ncoord, P.npairs = self.natoms, self.ncoord, self.npairs
        P.nsp, P.nk, P.nshell = self.nsp, self.nk, self.nshell
        P.iidx, P.jidx = N.dptr(self.d_i), N.dptr(self.d_j)
        P.shift = N.dptr(self.d_shift.contiguous())
        P.shell, P.sig2 = N.dptr(self.d_shell), N.dptr(self.d_sig2.contiguous())
        P.ftab, P.dtab = N.dptr(self.d_f), N.dptr(self.d_delta)
        P.lamtab, P.ktab = N.dptr(self.d_lam), N.dptr(self.d_k)
        P.drtab, P.c3tab, P.s2tab = N.dptr(self.d_dr), N.dptr(self.d_c3), N.dptr(self.d_s2tab)
        P.s02 = self.s02
        return P

    def distances(self, pos):
        """pos (nconf, natoms, 3) device tensor -> (r, evec)."""
        import torch
        pos = _dev(pos, torch.float64)
        nconf = pos.shape[0]
        r = torch.empty((nconf, self.npairs), dtype=torch.float64, device="cuda")
        ev = torch.empty((nconf, self.npairs, 3), dtype=torch.float64, device="cuda")
        N.call("chx_compute_r", N.ptr(pos), N.ptr(self.d_i), N.ptr(self.d_j),
               N.ptr(self.d_shift.contiguous()), N.ptr(r), N.ptr(ev), self.npairs, self.natoms,
               nconf, N.stream())
        return r, ev

    def ptypes(self, species):
        import torch
        species = _dev(species, torch.int32)
        nconf = species.shape[0]
        pt = torch.empty((nconf, self.npairs), dtype=torch.int32, device="cuda")
        N.call("chx_build_ptype", N.ptr(species), N.ptr(self.d_i), N.ptr(self.d_j), N.ptr(pt),
               self.npairs, self.natoms, nconf, self.nsp, N.stream())
        return pt

    # ---------------------------------------------------------------- forward
    def chi(self, pos, species, r=None, ptype=None, normalise=True, precision=FP64):
        """Discrete-species chi (nconf, nsp, nk); pos (nconf, natoms, 3),
        species (nconf, natoms) int32."""
        import torch
        pos = _dev(pos, torch.float64)
        species = _dev(species, torch.int32)
        nconf = pos.shape[0]
        chi = torch.empty((nconf, self.nsp, self.nk), dtype=torch.float64, device="cuda")
        if r is not None or ptype is not None:
            if r is None:
                r, _ = self.distances(pos)
            if ptype is None:
                ptype = self.ptypes(species)
            N.call("chx_chi_forward", N.ptr(r), N.ptr(ptype), N.ptr(self.d_shell),
                   N.ptr(self.d_sig2.contiguous()), N.ptr(self.d_f), N.ptr(self.d_delta),
                   N.ptr(self.d_lam), N.ptr(self.d_k), N.ptr(self.d_dr), N.ptr(self.d_c3),
                   N.ptr(self.d_s2tab), N.ptr(chi), self.npairs, self.nk, nconf, self.s02,
                   self.nsp, N.stream())
        else:
            self.chi_full(pos, species, precision=precision, out=chi)
        if normalise:
            cnt = torch.stack([(species == s).sum(dim=1) for s in range(self.nsp)], dim=1)
            chi /= cnt.clamp(min=1).to(torch.float64)[:, :, None]
        return chi

    def chi_full(self, pos, species, precision=FP64, out=None, max_scratch=1 << 30,
                 check=True):
        """Unnormalised path sum of every configuration (chx_chi_full),
        batched so the pair-record scratch stays under max_scratch bytes.
        With check (the default) the device error word of each batch is read
        back (one synchronisation) and a set word raises ChxError; a failed
        batch's chi is NaN either way."""
        import torch
        nconf = pos.shape[0]
        if out is None:
            out = torch.empty((nconf, self.nsp, self.nk), dtype=torch.float64, device="cuda")
        P = self.pairs_desc()
        per = max(1, int(max_scratch // max(1, self.npairs * 40)))
        words = []
        for c0 in range(0, nconf, per):
            c1 = min(nconf, c0 + per)
            n = c1 - c0
            need = int(N.lib().chx_chi_full_scratch_bytes(N.C.byref(P), n))
            scr = torch.empty(need, dtype=torch.uint8, device="cuda")
            N.call("chx_chi_full", N.C.byref(P), N.ptr(pos[c0:c1].contiguous()),
                   N.ptr(species[c0:c1].contiguous()), n, int(precision),
                   N.ptr(out[c0:c1]), N.ptr(scr), need, N.stream())
            if check:   # the error word: the int32 at need - 256
                words.append(scr[need - 256:need - 252].view(torch.int32))
        if words:
            w = int(torch.cat(words).max().item())
            if w:
                raise N.ChxError(f"chx_chi_full: device error word {w:#x} (an index, species "
                                 f"or shell out of range, or a bulk-copy wait that ran out)")
        return out


def _dev(x, dtype):
    import torch
    if isinstance(x, torch.Tensor):
        return x.to("cuda", dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x))).to("cuda", dtype)
