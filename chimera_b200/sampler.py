"""Parallel-tempering RMC on the device (methods/method_a_rmc.py).

`Ladders` owns the device state of a batch of independent temperature
ladders that share a species count: per ladder its supercell topology, tables,
transform, target and rungs; per replica slot its species, positions, chi(k),
chi^2, MS entry counts and best state. One `chx_sampler_step` launch advances
every slot of every ladder by one proposal; temperatures are exchanged by
permuting the rung <-> slot maps.

`RMCSampler` is the reference class's interface (constructor keywords,
init_state / step / replica_exchange / adapt / run / best / posterior_wc and
the attributes fitrun reads) on one ladder. With `reproduce=True` (default)
it consumes the reference's random streams: the proposal splitmix64 keyed
(seed, step, rung) on the device, the acceptance uniforms of
numpy PCG64(seed).random per step (the reference's `cp_rng`), and the
replica exchange decided on the host with a second PCG64(seed) exactly as
method_a_rmc.py:332-373 draws it. With `reproduce=False` the exchange is
decided on the device and whole blocks of steps replay as CUDA graphs.

`BatchedSampler` runs many ladders (sample positions, series points, uneven
supercells) in one launch per step under CUDA graphs, with periodic FP64
re-anchoring of the running chi (every `reanchor_every` accepted moves).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _native as N
from .forward import FP64, FP32C

KB_EV = 8.617333262e-5
MAX_BLOCK = 256          # steps per launch at most (rows of the accept log)


def _host(x):
    try:
        import torch
        if isinstance(x, torch.Tensor):
            return x.detach().cpu().numpy()
    except ImportError:
        pass
    return np.asarray(x)


def _fp32_rows(t):
    """FP32 copy of a (rows, nk) FP64 table with the row stride rounded up to
    a multiple of 4 (zero columns past nk), the layout of the step kernel's
    FP32 tables: it reads k points in 16-byte groups of four."""
    import torch
    rows, nk = t.shape
    out = torch.zeros((rows, (nk + 3) & ~3), dtype=torch.float32, device=t.device)
    out[:, :nk] = t
    return out


def _bf16_bits(x):
    """Round float32 values to BF16 (nearest, ties to even): the bit patterns
    (uint16) and the rounded values (float32)."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint32)
    return r.astype(np.uint16), (r << 16).view(np.float32)


def transform_fragments(f, win):
    """The fit-window transform W^T as split-BF16 A operands of mma m16n8k16
    (row-major A, the fragment layout of the PTX ISA): rows 2q (re) and
    2q + 1 (im) of window bin q, columns the ncoef taps of the shared tap run,
    entries norm * (cos, -sin)(2 pi n m_q / nfft), n = n0 + tap; hi = BF16(W),
    lo = BF16(W - hi). Returns (uint32 array [2][mt][kt][32][4], mt, kt)."""
    ncoef, nfft = int(f["ncoef"]), int(f["nfft"])
    win = np.asarray(win, np.int64)
    n = int(f["n0"][0]) + np.arange(ncoef)
    ph = (np.outer(win, n) % nfft).astype(np.float64) * (2.0 * np.pi / nfft)
    Wt = np.zeros((2 * win.size, ncoef))
    Wt[0::2] = np.cos(ph) * f["norm"]
    Wt[1::2] = -np.sin(ph) * f["norm"]
    mt, kt = -(-Wt.shape[0] // 16), -(-ncoef // 16)
    Wp = np.zeros((mt * 16, kt * 16), np.float32)
    Wp[:Wt.shape[0], :ncoef] = Wt
    hi_bits, hi = _bf16_bits(Wp)
    lo_bits, _ = _bf16_bits(Wp - hi)
    lane = np.arange(32)
    gid, tig = lane >> 2, lane & 3
    out = np.zeros((2, mt, kt, 32, 4), np.uint32)
    for part, bits in enumerate((hi_bits, lo_bits)):
        B = bits.astype(np.uint32).reshape(mt, 16, kt, 16).transpose(0, 2, 1, 3)  # [mt][kt][r][c]
        for r in range(4):
            row = gid + 8 * (r & 1)
            col = tig * 2 + 8 * (r >> 1)
            e0 = B[:, :, row, col]          # (mt, kt, 32)
            e1 = B[:, :, row, col + 1]
            out[part, :, :, :, r] = e0 | (e1 << 16)
    return out, mt, kt


def _window_gain_diag(f, win, sm, nsp, nk):
    """(nsp, nk): per edge e the diagonal of G_e = B_e W B_e^H, B_e the map
    from the edge's normalised chi(k) (nk) to its channels' chi(R) on the fit
    bins (resample, window x k^w, transform: the set-up f of _ft_setup) and W
    the weights 1 / sigma^2 (sm, (nchan, nwin)); G_kk is the weighted chi(R)
    norm^2 that a unit change at k alone produces."""
    nkw = f["nkw"]
    n = f["n0"][0] + np.arange(f["ncoef"])
    win = np.asarray(win, np.int64)
    z = np.exp(-2j * np.pi * ((np.outer(n, win) % f["nfft"]) / f["nfft"])) * f["norm"]
    out = np.zeros((nsp, nk))
    for e in range(nsp):
        for c in range(e * nkw, (e + 1) * nkw):
            B = np.zeros((nk, win.size), complex)
            wt = f["w"][c][:, None] * z
            np.add.at(B, f["idx"][c], (1.0 - f["frac"][c])[:, None] * wt)
            np.add.at(B, np.minimum(f["idx"][c] + 1, nk - 1), f["frac"][c][:, None] * wt)
            out[e] += (np.abs(B) ** 2 / np.asarray(sm[c], float)[None, :] ** 2).sum(1)
    return np.ascontiguousarray(out)


def torch_cat_host(ts):
    """Concatenate device tensors along dim 0 and bring them to the host."""
    import torch
    return torch.cat([t.reshape(t.shape[0], -1) for t in ts]).cpu().numpy()


def _on_device(x, dtype):
    """x as a contiguous CUDA tensor of dtype (one host->device copy, none
    for a device tensor of that type)."""
    import torch
    if isinstance(x, torch.Tensor):
        return x.to("cuda", dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(x)).to("cuda", dtype)


def _ft_setup(ft, nsp):
    """Per-channel window coefficients of a channel set (fourier.EdgeTransforms,
    the reference's chimera/multift.py adapter run through the cupy import
    shim, or one FourierTransform): n0, idx, frac, w padded to a common
    length."""
    fts = getattr(ft, "fts", None) or [ft]
    chan_edge = np.asarray(getattr(ft, "chan_edge", np.arange(len(fts))), np.int32)
    nkw = len(fts) // nsp
    assert nkw * nsp == len(fts), f"{len(fts)} channels do not divide into {nsp} edges"
    assert np.array_equal(chan_edge, np.repeat(np.arange(nsp), nkw)), \
        "channels must be ordered edge-major"
    # every channel's non-zero taps, placed on one shared run of the uniform
    # grid [n0, n0 + ncoef) (zero weight outside a channel's own window)
    spans = []
    for f in fts:
        wt = _host(f._w) * _host(f._inside)
        nz = np.nonzero(wt)[0]
        spans.append((int(nz[0]), int(nz[-1]) + 1) if nz.size else (0, 1))
    n0u = min(a for a, _ in spans)
    ncoef = max(b for _, b in spans) - n0u
    I = np.zeros((len(fts), ncoef), np.int32)
    F = np.zeros((len(fts), ncoef))
    W = np.zeros((len(fts), ncoef))
    for c, f in enumerate(fts):
        idx, frac = _host(f._idx), _host(f._frac)
        wt = _host(f._w) * _host(f._inside)
        a, b = spans[c]
        I[c, a - n0u:b - n0u] = idx[a:b]
        F[c, a - n0u:b - n0u] = frac[a:b]
        W[c, a - n0u:b - n0u] = wt[a:b]
    n0 = np.full(len(fts), n0u, np.int32)
    nfft = int(fts[0].nfft)
    norm = float(fts[0]._norm)
    extra = getattr(ft, "chi_extra", None)
    return dict(nchan=len(fts), nkw=nkw, n0=n0, idx=I, frac=F, w=W, ncoef=ncoef, nfft=nfft,
                norm=norm, extra=None if extra is None else _host(extra))


class LadderSpec:
    """Inputs of one temperature ladder (everything RMCSampler takes)."""

    def __init__(self, fm, ft, target, mask, sigma_R, nrep=48, tmin=0.02, tmax=5.0, seed=0,
                 swap_frac=0.75, disp_sigma=0.015, max_disp=0.30, profile_scale=True,
                 energy_prior=None, ms_library=None):
        self.fm, self.ft = fm, ft
        self.target = np.asarray(target)
        self.mask = np.asarray(mask, bool)
        self.sigma_R = np.asarray(sigma_R, float)
        self.nrep, self.tmin, self.tmax, self.seed = int(nrep), tmin, tmax, int(seed)
        self.swap_frac, self.disp_sigma, self.max_disp = swap_frac, disp_sigma, max_disp
        self.profile_scale = bool(profile_scale)
        self.energy_prior = energy_prior
        # the package's MS object, or the reference's own SupercellMS adopted
        # onto the forward model's supercell
        from .mspaths import SupercellMS
        self.ms = SupercellMS.adopt(ms_library, fm.cell) if ms_library is not None else None


class Ladders:
    """Device state and descriptors of a batch of ladders (see module doc)."""

    # FP32C: keep each slot's FP64 chi(R) and transform only a move's change
    # (xr of chx_ladder_t), with the near-tie FP64 re-check
    delta_transform = True
    # the near-tie test's relative RMS rounding of the change's transform
    # (split BF16, three products: ~3e-6 per element); 0 turns the test off
    tie_eps = 5e-6
    # FP32C with the kept chi(R): the change's window transform as split-BF16
    # tensor-core products (ft_frag of chx_ladder_t) instead of the FP32 DFT
    tc_transform = True

    def __init__(self, specs, precision=FP64, use_table=True, threads=256, min_blocks=3):
        import torch
        N.require_cuda()
        self.threads, self.min_blocks = int(threads), int(min_blocks)
        self.torch = torch
        self.specs = list(specs)
        self.precision = int(precision)
        self.nsp = int(self.specs[0].fm.nsp)
        assert all(s.fm.nsp == self.nsp for s in self.specs), "one species count per batch"
        self.nladders = len(self.specs)
        self.nslots = sum(s.nrep for s in self.specs)
        self.use_table = bool(use_table) and self.precision != FP64
        self.host = (N.Ladder * self.nladders)()
        self.keep = []                      # device tensors the descriptors point to
        self.bufs = []                      # per-ladder dict of named tensors
        slot0 = 0
        slot_ladder = []
        for li, s in enumerate(self.specs):
            self.bufs.append(self._build_ladder(li, s, slot0))
            slot_ladder += [li] * s.nrep
            slot0 += s.nrep
        self.slot_ladder = N.to_dev(np.array(slot_ladder, np.int32))
        self.stepc = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.ticket = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.err = torch.zeros(1, dtype=torch.int32, device="cuda")
        self._upload()

    # ------------------------------------------------------------ building
    def _t(self, a, dtype=None):
        t = N.to_dev(a, dtype)
        self.keep.append(t)
        return t

    def _supercell(self, fm):
        """Per-supercell device data shared by every ladder on the same
        ForwardModel: reverse pair index, ideal sites, shifts, sigma^2, the
        pairs that may use the (shell, type) table and the shell radii."""
        # kept on the forward model, so every sampler built on it shares the
        # host-side work and the device arrays
        # (an entry is valid while the model's geometry and cumulant tables
        # are the same tensors: set_dr/set_c3/set_sig2_types replace them)
        cache = fm.__dict__.setdefault("_ladder_cell_cache", {})
        key = "cell"
        src = (fm.d_shift, fm.d_sig2, fm.d_dr, fm.d_c3, fm.d_s2tab)
        if key in cache and all(a is b for a, b in zip(cache[key]["src"], src)):
            return cache[key]
        i_np, j_np = fm.i_idx, fm.j_idx
        natoms = fm.natoms
        z = np.bincount(i_np, minlength=natoms)
        assert z.min() == z.max(), "expected uniform coordination"
        ncoord = int(z[0])
        assert np.array_equal(i_np, np.repeat(np.arange(natoms), ncoord)), \
            "pairs must be i-major (pair p = i * ncoord + o)"
        from .lattice import build_reverse_index
        rev = build_reverse_index(i_np, j_np, natoms)
        ideal = np.ascontiguousarray(fm.cell.ideal, np.float64)
        shift = _host(fm.d_shift).astype(np.float64)
        sig2 = _host(fm.d_sig2).astype(np.float64)
        shell = fm.shell
        d0 = np.linalg.norm((ideal[j_np] + shift) - ideal[i_np], axis=1)
        first = np.array([np.argmax(shell == q) for q in range(fm.nshell)])
        r_shell, s2_shell = d0[first], sig2[first]
        pair_tab = ((np.abs(d0 - r_shell[shell]) <= 1e-12 * r_shell[shell])
                    & (sig2 == s2_shell[shell]))
        pair_tab = (pair_tab & pair_tab[rev]).astype(np.uint8)   # a pair and its reverse agree
        c = dict(ncoord=ncoord, r_shell=r_shell, s2_shell=s2_shell, src=src,
                 dev=dict(rev=self._t(rev), ideal=self._t(ideal), shift=self._t(shift),
                          sig2=self._t(sig2), pair_tab=self._t(pair_tab)))
        cache[key] = c
        return c

    def _build_ladder(self, li, s, slot0):
        torch = self.torch
        fm = s.fm
        L = self.host[li]
        nsp, nk, nrep = self.nsp, fm.nk, s.nrep
        natoms = fm.natoms
        cell = self._supercell(fm)
        ncoord, r_shell, s2_shell = cell["ncoord"], cell["r_shell"], cell["s2_shell"]
        b = dict(cell["dev"])
        L.natoms, L.ncoord, L.npairs, L.nshell, L.nsp, L.nk = (natoms, ncoord, fm.npairs,
                                                              fm.nshell, nsp, nk)
        L.iidx, L.jidx, L.rev = N.dptr(fm.d_i), N.dptr(fm.d_j), N.dptr(b["rev"])
        L.shift, L.shell, L.sig2 = N.dptr(b["shift"]), N.dptr(fm.d_shell), N.dptr(b["sig2"])
        L.pair_tab, L.ideal = N.dptr(b["pair_tab"]), N.dptr(b["ideal"])
        L.ftab, L.dtab, L.lamtab, L.ktab = (N.dptr(fm.d_f), N.dptr(fm.d_delta),
                                            N.dptr(fm.d_lam), N.dptr(fm.d_k))
        L.drtab, L.c3tab, L.s2tab = N.dptr(fm.d_dr), N.dptr(fm.d_c3), N.dptr(fm.d_s2tab)
        self.keep += [fm.d_i, fm.d_j, fm.d_shell, fm.d_f, fm.d_delta, fm.d_lam, fm.d_k,
                      fm.d_dr, fm.d_c3, fm.d_s2tab]
        L.s02 = fm.s02
        if self.use_table:
            if "sstab" not in cell:      # the (shell, type) table, once per supercell
                cell["sstab"] = torch.empty((fm.nshell * nsp * nsp, nk), dtype=torch.float64,
                                            device="cuda")
                self.keep.append(cell["sstab"])
                L.sstab = N.dptr(cell["sstab"])
                rs, ss = self._t(r_shell), self._t(s2_shell)
                N.call("chx_shell_table", C.byref(L), N.ptr(rs), N.ptr(ss),
                       N.ptr(cell["sstab"]), N.stream())
                cell["sstab32"] = _fp32_rows(cell["sstab"])
                self.keep.append(cell["sstab32"])
            b["sstab"], b["sstab32"] = cell["sstab"], cell["sstab32"]
            L.sstab, L.sstab32 = N.dptr(b["sstab"]), N.dptr(b["sstab32"])
        else:
            L.sstab, L.sstab32 = 0, 0
        # exact multiple scattering
        ms = s.ms
        if ms is not None:
            d = ms.paths.device(("tpl", "nbr"))
            L.ms_nblk, L.ms_M, L.ms_D = ms.nblk, ms.paths.tpl.shape[0], ms.paths.D
            L.ms_tpl, L.ms_nbr, L.ms_T = N.dptr(d["tpl"]), N.dptr(d["nbr"]), N.dptr(ms.T)
            self.keep += [d["tpl"], d["nbr"], ms.T]
            if self.precision != FP64:
                key = ("msT32", id(ms))
                if key not in cell:
                    cell[key] = _fp32_rows(ms.T)
                    self.keep.append(cell[key])
                b["msT32"] = cell[key]
                L.ms_T32 = N.dptr(b["msT32"])
            else:
                L.ms_T32 = 0
        else:
            L.ms_nblk, L.ms_M, L.ms_D, L.ms_tpl, L.ms_nbr, L.ms_T, L.ms_T32 = 0, 0, 0, 0, 0, 0, 0
        # pair-interaction prior (method_a_rmc.py:147-157)
        if s.energy_prior is not None:
            V, T_ann = s.energy_prior
            V = np.asarray(V, float)
            tab = np.zeros((fm.nshell, nsp * nsp))
            m = min(fm.nshell, V.shape[0])
            tab[:m] = 0.5 * V[:m].reshape(m, nsp * nsp)
            b["etab"] = self._t(tab.reshape(-1))
            L.etab = N.dptr(b["etab"])
            L.energy_beta = 1.0 / (KB_EV * float(T_ann))
        else:
            L.etab, L.energy_beta = 0, 0.0
        # transform and target (the set-up once per transform object)
        try:        # kept on the transform object when it allows attributes
            fcache = s.ft.__dict__.setdefault("_ladder_ft_cache", {})
        except AttributeError:
            fcache = self.__dict__.setdefault("_ft_cache", {})
        if id(s.ft) not in fcache:
            f = _ft_setup(s.ft, nsp)
            fcache[id(s.ft)] = (s.ft, f, dict(ft_n0=self._t(f["n0"]), ft_idx=self._t(f["idx"]),
                                              ft_frac=self._t(f["frac"]), ft_w=self._t(f["w"])))
        f = fcache[id(s.ft)][1]
        b.update(fcache[id(s.ft)][2])
        win = np.nonzero(s.mask)[0].astype(np.int32)
        cplx = bool(np.iscomplexobj(s.target))
        tm = np.ascontiguousarray(s.target[:, s.mask])
        sm = np.ascontiguousarray(s.sigma_R[:, s.mask], np.float64)
        b.update(win=self._t(win),
                 tm_re=self._t(np.ascontiguousarray(tm.real, np.float64)),
                 tm_im=self._t(np.ascontiguousarray(tm.imag if cplx else np.zeros(tm.shape),
                                                    np.float64)),
                 sm=self._t(sm), w2=self._t(1.0 / (sm * sm)),
                 tnorm=self._t(((np.abs(tm) ** 2) / (sm * sm)).sum(1)))
        if f["extra"] is not None:
            b["extra"] = self._t(np.ascontiguousarray(f["extra"], np.float64))
        L.nchan, L.nkw, L.nwin, L.nfft, L.ncoef = (f["nchan"], f["nkw"], int(win.size),
                                                  f["nfft"], f["ncoef"])
        L.ft_n0, L.ft_idx, L.ft_frac, L.ft_w = (N.dptr(b["ft_n0"]), N.dptr(b["ft_idx"]),
                                                N.dptr(b["ft_frac"]), N.dptr(b["ft_w"]))
        L.win_bin, L.ft_norm = N.dptr(b["win"]), f["norm"]
        L.chi_extra = N.dptr(b.get("extra"))
        L.tm_re, L.tm_im, L.sm = N.dptr(b["tm_re"]), N.dptr(b["tm_im"]), N.dptr(b["sm"])
        L.w2, L.tnorm = N.dptr(b["w2"]), N.dptr(b["tnorm"])
        L.cplx, L.profile = int(cplx), int(s.profile_scale)
        self.nfit_of = getattr(self, "nfit_of", []) + [int(s.mask.sum()) * f["nchan"] * (2 if cplx else 1)]
        L.nfit = float(self.nfit_of[-1])
        # sampler constants
        L.seed = s.seed & (2 ** 64 - 1)
        L.swap_frac, L.disp_sigma, L.max_disp = s.swap_frac, s.disp_sigma, s.max_disp
        L.nrep, L.slot0 = nrep, slot0
        beta = 1.0 / np.geomspace(s.tmin, s.tmax, nrep)
        b["beta"] = self._t(beta)
        L.beta_rung = N.dptr(b["beta"])
        L.u_stream, L.u_steps = 0, 0
        # state
        z32 = lambda *sh: torch.zeros(sh, dtype=torch.int32, device="cuda")
        f64 = lambda *sh: torch.zeros(sh, dtype=torch.float64, device="cuda")
        b.update(species=z32(nrep, natoms), pos=f64(nrep, natoms, 3),
                 moved=torch.zeros((nrep, natoms), dtype=torch.uint8, device="cuda"),
                 chi=f64(nrep, nsp, nk), chi2=f64(nrep), count=f64(nrep, nsp),
                 rung_of=z32(nrep), slot_of=z32(nrep), best_chi2=f64(nrep),
                 best_sp=z32(nrep, natoms), best_pos=f64(nrep, natoms, 3),
                 ms_C=z32(nrep, ms.nent if ms is not None else 1),
                 acc=torch.zeros(nrep, dtype=torch.uint8, device="cuda"),
                 acc_log=torch.zeros((MAX_BLOCK, nrep), dtype=torch.uint8, device="cuda"),
                 n_acc=z32(nrep),
                 exch_att=z32(max(nrep, 1)), exch_acc=z32(max(nrep, 1)),
                 best_stale=torch.ones(nrep, dtype=torch.uint8, device="cuda"))
        for key in ("species", "pos", "moved", "chi", "chi2", "count", "rung_of", "slot_of",
                    "best_chi2", "best_sp", "best_pos", "ms_C", "acc", "acc_log", "n_acc",
                    "exch_att", "exch_acc", "best_stale"):
            self.keep.append(b[key])
        L.species, L.pos, L.moved, L.chi = (N.dptr(b["species"]), N.dptr(b["pos"]),
                                            N.dptr(b["moved"]), N.dptr(b["chi"]))
        L.chi2, L.count, L.rung_of, L.slot_of = (N.dptr(b["chi2"]), N.dptr(b["count"]),
                                                 N.dptr(b["rung_of"]), N.dptr(b["slot_of"]))
        L.best_chi2, L.best_sp, L.best_pos = (N.dptr(b["best_chi2"]), N.dptr(b["best_sp"]),
                                              N.dptr(b["best_pos"]))
        L.ms_C, L.acc_rung, L.n_acc = N.dptr(b["ms_C"]), N.dptr(b["acc"]), N.dptr(b["n_acc"])
        L.acc_log = N.dptr(b["acc_log"])
        L.exch_att, L.exch_acc = N.dptr(b["exch_att"]), N.dptr(b["exch_acc"])
        L.best_stale = N.dptr(b["best_stale"])
        # FP32C: the slots' FP64 chi(R) on the fit window (the step transforms
        # a move's change alone) and the near-tie FP64 re-check
        if self.precision != FP64 and self.delta_transform:
            b["xr"] = torch.zeros((nrep, f["nchan"], int(win.size), 2), dtype=torch.float64,
                                  device="cuda")
            b["tie_stat"] = torch.zeros((nrep, 2), dtype=torch.float64, device="cuda")
            b["xs"] = torch.ones((nrep, nsp), dtype=torch.float64, device="cuda")
            self.keep += [b["xr"], b["tie_stat"], b["xs"]]
            L.xs = N.dptr(b["xs"])
            L.xr, L.tie_stat, L.tie_eps = N.dptr(b["xr"]), N.dptr(b["tie_stat"]), self.tie_eps
            # the FP32 terms' share of the near-tie bound: the transform's
            # per-k gain (diagonal of B W B^H per edge)
            if self.tie_eps > 0:
                b["tie_gdiag"] = self._t(_window_gain_diag(f, win, sm, nsp, nk))
                L.tie_gdiag = N.dptr(b["tie_gdiag"])
            else:
                L.tie_gdiag = 0
            # the change's transform on the tensor cores (split BF16)
            if self.tc_transform:
                key = tuple(win.tolist())
                fc = fcache.setdefault(("ft_frag", id(s.ft)), {})
                if key not in fc:
                    frag, mt, kt = transform_fragments(f, win)
                    fc[key] = (self._t(frag.reshape(-1).view(np.int32)), mt, kt)
                b["ft_frag"], L.ft_mt, L.ft_kt = fc[key]
                b["ft_tiles"] = (L.ft_mt, L.ft_kt)
                L.ft_frag = N.dptr(b["ft_frag"])
            else:
                L.ft_frag, L.ft_mt, L.ft_kt = 0, 0, 0
        else:
            L.xr, L.tie_stat, L.tie_eps = 0, 0, 0.0
            L.tie_gdiag, L.xs = 0, 0
            L.ft_frag, L.ft_mt, L.ft_kt = 0, 0, 0
        b["beta_host"] = beta
        b["cplx"] = cplx
        return b

    def _upload(self):
        """Copy the host descriptors to the device, into the same buffer once
        it exists (so a captured graph keeps a valid address)."""
        import torch
        raw = bytes(C.string_at(C.addressof(self.host), C.sizeof(self.host)))
        src = torch.frombuffer(bytearray(raw), dtype=torch.uint8)
        if getattr(self, "d_ladders", None) is None or self.d_ladders.numel() != src.numel():
            self.d_ladders = src.to("cuda")
        else:
            self.d_ladders.copy_(src)
        return self.d_ladders

    def has_tc_transform(self):
        """Whether the ladders carry the tensor-core operands of the change's
        window transform (FP32C with the kept chi(R))."""
        return any("ft_frag" in b for b in self.bufs)

    def set_transform(self, tensor_cores):
        """Transform a move's change with the split-BF16 tensor-core products
        (True) or the FP32 rotation DFT (False); FP32C with the kept chi(R).
        Takes effect for launches made (or graphs captured) after the call."""
        for li, b in enumerate(self.bufs):
            if "ft_frag" not in b:
                continue
            L = self.host[li]
            if tensor_cores:
                L.ft_frag = N.dptr(b["ft_frag"])
                L.ft_mt, L.ft_kt = b["ft_tiles"]
            else:
                L.ft_frag, L.ft_mt, L.ft_kt = 0, 0, 0
        self._upload()

    def set_field(self, li, name, value):
        setattr(self.host[li], name, value)
        self._upload()

    # --------------------------------------------------------------- state
    def init_state(self, li, species0, pos0, stream_species=None, defer=False):
        """Every rung of ladder li starts from (species0, pos0). With `defer`
        (and the shell table on) the FP64 start chi is left to one
        chx_reanchor launch over every slot of the batch (`anchor_pending`)
        instead of a full path sum per ladder; the two agree to rounding."""
        torch = self.torch
        s, b = self.specs[li], self.bufs[li]
        fm = s.fm
        nrep = s.nrep
        # one copy of the start state crosses to the device (a device tensor
        # is used as it is) and is broadcast to every rung there
        dsp = _on_device(species0, torch.int32)
        dpos = _on_device(pos0, torch.float64)
        b["species"].copy_(dsp[None].expand(nrep, -1))
        b["pos"].copy_(dpos[None].expand(nrep, -1, -1))
        ideal = self._supercell(fm)["dev"]["ideal"]
        b["moved"].copy_((dpos != ideal).any(dim=-1).to(torch.uint8)[None].expand(nrep, -1))
        # every rung starts from the same configuration: evaluate it once
        if s.ms is not None:
            C_ = s.ms.counts(b["species"][:1].contiguous())
            b["ms_C"].copy_(C_.expand(nrep, -1))
        if defer and self.use_table:
            b["chi"].zero_()
            self.__dict__.setdefault("_pending", set()).add(li)
        else:
            chi = fm.chi_full(b["pos"][:1].contiguous(), b["species"][:1].contiguous(),
                              precision=FP64)
            if s.ms is not None:
                chi = chi + s.ms.chi_of(C_)
            b["chi"].copy_(chi.expand(nrep, -1, -1))
        cnt = torch.bincount(dsp.long(), minlength=self.nsp)[:self.nsp].to(torch.float64)
        b["count"].copy_(cnt[None].expand(nrep, -1))
        b["rung_of"].copy_(torch.arange(nrep, dtype=torch.int32))
        b["slot_of"].copy_(torch.arange(nrep, dtype=torch.int32))
        b["acc"].zero_()
        b["n_acc"].zero_()
        b["exch_att"].zero_()
        b["exch_acc"].zero_()

    def eval_chi2(self, chi_in=None, count_in=None):
        """chi^2 of every slot (nslots) by the step's own transform."""
        torch = self.torch
        out = torch.empty(self.nslots, dtype=torch.float64, device="cuda")
        N.call("chx_eval_chi2", N.ptr(self.d_ladders), C.byref(self.host), self.nladders,
               N.ptr(self.slot_ladder), self.nslots, self.precision,
               N.ptr(chi_in) if chi_in is not None else None,
               N.ptr(count_in) if count_in is not None else None, N.ptr(out), N.stream())
        return out

    def refresh_chi2(self, reset_best=False):
        c2 = self.eval_chi2()
        for li, b in enumerate(self.bufs):
            s0 = self.host[li].slot0
            b["chi2"].copy_(c2[s0:s0 + self.specs[li].nrep])
            if reset_best:
                b["best_chi2"].copy_(b["chi2"])
                b["best_sp"].copy_(b["species"])
                b["best_pos"].copy_(b["pos"])
                b["best_stale"].zero_()

    def reanchor(self, mask=None):
        """Replace the running chi of the slots in `mask` (a (nslots,) bool
        array; None: all) by an FP64 recompute from their species, positions
        and exact MS counts, reset their accepted-move counters, and refresh
        chi^2. With the (shell, type) table this is one chx_reanchor launch
        (pair-count form); otherwise the full FP64 path sum."""
        torch = self.torch
        if self.use_table:
            m = None if mask is None else torch.as_tensor(mask).to("cuda", torch.uint8).contiguous()
            need = int(N.lib().chx_reanchor_scratch_bytes(C.byref(self.host), self.nladders,
                                                          self.nslots))
            scr = torch.empty(need, dtype=torch.uint8, device="cuda")
            N.call("chx_reanchor", N.ptr(self.d_ladders), C.byref(self.host), self.nladders,
                   N.ptr(self.slot_ladder), self.nslots, N.ptr(m) if m is not None else None,
                   N.ptr(scr), need, N.ptr(self.err), N.stream())
            # chi^2 (and the FP32C chi(R)) of the re-anchored slots only
            N.call("chx_refresh_chi2", N.ptr(self.d_ladders), C.byref(self.host), self.nladders,
                   N.ptr(self.slot_ladder), self.nslots, self.precision,
                   N.ptr(m) if m is not None else None, N.stream())
            self._reanchor_keep = (m, scr)      # alive until the launches have run
            return
        else:
            for s, b in zip(self.specs, self.bufs):
                chi = s.fm.chi_full(b["pos"], b["species"], precision=FP64)
                if s.ms is not None:
                    chi = chi + s.ms.chi_of(b["ms_C"])
                b["chi"].copy_(chi)
                b["n_acc"].zero_()
        self.refresh_chi2()

    def anchor_pending(self):
        """FP64 start chi of the ladders initialised with `defer`: one
        chx_reanchor launch over their slots (pair-count form)."""
        pend = self.__dict__.pop("_pending", set())
        if not pend:
            return
        mask = np.zeros(self.nslots, bool)
        for li in pend:
            s0 = self.host[li].slot0
            mask[s0:s0 + self.specs[li].nrep] = True
        self.reanchor(mask)

    def reanchor_due(self, every):
        """Re-anchor, inside the current stream (capturable), every slot
        whose accepted-move counter reached `every`: the device decides
        (chx_reanchor_due), recomputes those slots' chi in FP64, refreshes
        their chi^2 and counts them in `self.reanchor_count`."""
        torch = self.torch
        if getattr(self, "due", None) is None:
            self.due = torch.zeros(self.nslots, dtype=torch.uint8, device="cuda")
            self.reanchor_count = torch.zeros(1, dtype=torch.int64, device="cuda")
            # at most this many slots per period (the rest follow a period
            # later); the batch workload averages about two
            self.max_due = min(self.nslots, int(getattr(self, "reanchor_cap", 8)))
            need = int(N.lib().chx_reanchor_scratch_bytes(C.byref(self.host), self.nladders,
                                                          self.max_due))
            self.ra_scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
        N.call("chx_reanchor_due", N.ptr(self.d_ladders), C.byref(self.host), self.nladders,
               N.ptr(self.slot_ladder), self.nslots, int(every), self.max_due, self.precision,
               N.ptr(self.due), N.ptr(self.reanchor_count), N.ptr(self.ra_scratch),
               int(self.ra_scratch.numel()), N.ptr(self.err), N.stream())

    def slot_reanchors(self):
        """Slots re-anchored on the device so far (chx_reanchor_due)."""
        rc = getattr(self, "reanchor_count", None)
        return 0 if rc is None else int(rc.item())

    def accepted_since_anchor(self):
        """(nslots,) accepted moves since each slot's last re-anchoring."""
        return self.torch.cat([b["n_acc"] for b in self.bufs])

    # --------------------------------------------------------------- steps
    def step(self, nsteps=1):
        """nsteps steps of every slot in one launch (nsteps <= MAX_BLOCK)."""
        assert 0 < nsteps <= MAX_BLOCK
        N.call("chx_sampler_step", N.ptr(self.d_ladders), C.byref(self.host), self.nladders,
               N.ptr(self.slot_ladder), self.nslots, self.precision, int(nsteps),
               self.threads, self.min_blocks, N.ptr(self.stepc), N.ptr(self.ticket),
               N.ptr(self.err), N.stream())

    def exchange_device(self):
        N.call("chx_replica_exchange", N.ptr(self.d_ladders), self.nladders, N.ptr(self.stepc),
               N.stream())

    def apply_exchange(self, li, order):
        o = N.to_dev(np.asarray(order, np.int32))
        N.call("chx_apply_exchange", N.ptr(self.d_ladders), li, N.ptr(o), N.stream())
        self._last_order = o                # keep alive until the launch has run

    def device_error(self):
        return int(self.err.item())

    # ------------------------------------------------ surrogate and swap log
    def feature_table(self, li):
        """Ladder li's (natoms, D) feature neighbourhoods (built once)."""
        b, L = self.bufs[li], self.host[li]
        if "feat_nbr" not in b:
            from .surrogate import feature_neighbours
            fm = self.specs[li].fm
            cell = self._supercell(fm)
            if "feat" not in cell:       # once per supercell
                nbr = feature_neighbours(_host(fm.cell.ideal), fm.i_idx, fm.j_idx,
                                         _host(fm.d_shift), L.ncoord)
                cell["feat"] = (nbr, self._t(nbr))
            b["feat_nbr_host"], b["feat_nbr"] = cell["feat"]
            L.feat_nbr, L.feat_D = N.dptr(b["feat_nbr"]), int(b["feat_nbr_host"].shape[1])
        return b["feat_nbr_host"]

    def _da_buffers(self, li):
        b = self.bufs[li]
        if "da_on" not in b:
            b["da_on"] = self._t(np.zeros(1, np.int32))
            b["da_stat"] = self._t(np.zeros((self.specs[li].nrep, 4)))
            L = self.host[li]
            L.da_on, L.da_stat = N.dptr(b["da_on"]), N.dptr(b["da_stat"])
        return b

    def attach_surrogate(self, sur, ladders=None, on=True):
        """Screen the swaps of the given ladders (default all) with `sur`
        (a surrogate.SwapSurrogate), screening on or off. Changes the step
        kernel's shared-memory plan: recapture graphs afterwards."""
        for li in (range(self.nladders) if ladders is None else ladders):
            self.feature_table(li)
            assert sur.D == self.host[li].feat_D and sur.nsp == self.nsp, "surrogate shape"
            b = self._da_buffers(li)
            b["da_on"].fill_(1 if on else 0)
            self.host[li].mlp = sur.device_ptr
        self._surrogate = sur
        self._upload()

    def detach_surrogate(self):
        for li in range(self.nladders):
            self.host[li].mlp = 0
        self._upload()

    def set_screening(self, li, on):
        """Switch ladder li's screen on or off (a device word: no re-plan,
        captured graphs stay valid)."""
        self._da_buffers(li)["da_on"].fill_(1 if on else 0)

    def screening_on(self):
        return [bool(int(b["da_on"].item())) if "da_on" in b else False for b in self.bufs]

    def tie_stats(self, reset=False):
        """(nladders, 2) summed over each ladder's slots: Metropolis tests
        re-decided with FP64 transforms (near ties), and decisions they
        changed (FP32C with the kept chi(R))."""
        out = np.zeros((self.nladders, 2))
        for li, b in enumerate(self.bufs):
            if "tie_stat" in b:
                out[li] = _host(b["tie_stat"]).sum(0)
                if reset:
                    b["tie_stat"].zero_()
        return out

    def da_stats(self, reset=False):
        """(nladders, 4) summed over each ladder's slots: moves screened,
        moves passed to the exact stage, moves accepted there, and the sum of
        the stage-2 acceptance probabilities of the passed moves."""
        out = np.zeros((self.nladders, 4))
        for li, b in enumerate(self.bufs):
            if "da_stat" in b:
                out[li] = _host(b["da_stat"]).sum(0)
                if reset:
                    b["da_stat"].zero_()
        return out

    def enable_log(self, cap, ladders=None):
        """Log the swaps of the given ladders (default all) that are evaluated
        exactly: features, sigma * d, ln beta, chain and step into a ring of
        `cap` entries each."""
        torch = self.torch
        for li in (range(self.nladders) if ladders is None else ladders):
            self.feature_table(li)
            b, L = self.bufs[li], self.host[li]
            b["log_codes"] = torch.zeros((int(cap), 2 * L.feat_D + 1), dtype=torch.uint8,
                                         device="cuda")
            b["log_y"] = torch.full((int(cap), 4), float("nan"), dtype=torch.float32,
                                    device="cuda")
            self.keep += [b["log_codes"], b["log_y"]]
            L.log_codes, L.log_y, L.log_cap = N.dptr(b["log_codes"]), N.dptr(b["log_y"]), int(cap)
        self._upload()

    def disable_log(self):
        for L in self.host:
            L.log_cap = 0
        self._upload()

    def swap_log(self, ladders=None, extra=False):
        """(codes, lnbeta, y) of the logged swaps (device tensors); with
        extra, also (chain, step) of each."""
        torch = self.torch
        cs, rows = [], []
        for li in (range(self.nladders) if ladders is None else ladders):
            b = self.bufs[li]
            if "log_y" not in b:
                continue
            ok = torch.isfinite(b["log_y"][:, 0])
            cs.append(b["log_codes"][ok])
            rows.append(b["log_y"][ok])
        y = torch.cat(rows)
        out = (torch.cat(cs), y[:, 1].contiguous(), y[:, 0].contiguous())
        return out + (y[:, 2].long(), y[:, 3].long()) if extra else out


class RMCSampler:
    """Device PT-RMC with the reference RMCSampler's interface."""

    def __init__(self, fm, ft, target, mask, sigma_R, nrep=48, tmin=0.02, tmax=5.0, seed=0,
                 swap_frac=0.75, disp_sigma=0.015, max_disp=0.30, nsp=None,
                 collect_after=None, collect_every=25, adapt_every=0, target_accept=0.35,
                 profile_scale=True, collect_beta=0.5, n_collect=4, energy_prior=None,
                 ms_library=None, precision=FP64, reproduce=True, use_table=True):
        self.fm, self.ft = fm, ft
        self.nsp = int(nsp) if nsp is not None else int(fm.nsp)
        self.nrep = int(nrep)
        self.collect_after = collect_after
        self.collect_every = int(collect_every)
        self.collect_beta = None if collect_beta is None else float(collect_beta)
        self.n_collect = int(n_collect)
        self.adapt_every = int(adapt_every)
        self.target_accept = float(target_accept)
        self.profile_scale = bool(profile_scale)
        self.samples = []
        self.seed = int(seed)
        self.rng = np.random.default_rng(seed)              # exchange stream
        self._u_gen = np.random.default_rng(seed)            # acceptance stream
        self.swap_frac, self.disp_sigma, self.max_disp = swap_frac, disp_sigma, max_disp
        self.reproduce = bool(reproduce)
        self.spec = LadderSpec(fm, ft, target, mask, sigma_R, nrep=nrep, tmin=tmin, tmax=tmax,
                               seed=seed, swap_frac=swap_frac, disp_sigma=disp_sigma,
                               max_disp=max_disp, profile_scale=profile_scale,
                               energy_prior=energy_prior, ms_library=ms_library)
        self.ms = self.spec.ms
        self.lad = Ladders([self.spec], precision=precision, use_table=use_table)
        self.b = self.lad.bufs[0]
        self.complex = self.b["cplx"]
        self.nfit = self.lad.nfit_of[0]
        self.natoms, self.npairs, self.nk = fm.natoms, fm.npairs, fm.nk
        self.exch_attempts = np.zeros(max(nrep - 1, 1))
        self.exch_accepted = np.zeros(max(nrep - 1, 1))
        self._u_host = np.zeros((0, self.nrep))
        self._stepc = 0

    # ------------------------------------------------------------ state
    def init_state(self, species0, pos0):
        self.lad.init_state(0, species0, pos0)
        self.lad.refresh_chi2(reset_best=True)

    def _ensure_uniforms(self, upto):
        """Acceptance uniforms for steps 1..upto, PCG64(seed).random(nrep)
        per step (the reference's cp_rng draws, method_a_rmc.py:284)."""
        if not self.reproduce or self._u_host.shape[0] >= upto:
            return
        grow = max(upto - self._u_host.shape[0], 1024)
        more = self._u_gen.random(grow * self.nrep).reshape(grow, self.nrep)
        self._u_host = np.concatenate([self._u_host, more])
        self._u_dev = N.to_dev(self._u_host)
        L = self.lad.host[0]
        L.u_stream, L.u_steps = N.dptr(self._u_dev), self._u_host.shape[0]
        self.lad._upload()

    @property
    def _rung_slots(self):
        return self.b["slot_of"].long()

    @property
    def chi2(self):
        """(nrep,) chi^2 by rung (device)."""
        return self.b["chi2"][self._rung_slots]

    @property
    def species(self):
        return self.b["species"][self._rung_slots]

    @property
    def pos(self):
        return self.b["pos"][self._rung_slots]

    @property
    def chi(self):
        return self.b["chi"][self._rung_slots]

    @property
    def beta(self):
        return self.b["beta"]

    @property
    def best_chi2(self):
        return self.b["best_chi2"]

    def scales(self, chi_un=None):
        raise NotImplementedError("profiled scales are evaluated inside the device step")

    # ------------------------------------------------------------ moves
    def step(self):
        """One proposal per rung; returns the accept flags by rung (device)."""
        self._stepc += 1
        self._ensure_uniforms(self._stepc)
        self.lad.step(1)
        return self.b["acc"].bool()

    def steps(self, n):
        """n proposals per rung in one launch; accept flags (n, nrep) by rung."""
        self._stepc += n
        self._ensure_uniforms(self._stepc)
        self.lad.step(n)
        return self.b["acc_log"][:n]

    def replica_exchange(self, return_rates=False):
        """Host-decided exchange on the reference's PCG64 stream
        (method_a_rmc.py:332-373); the state stays put, the rungs move."""
        c2 = _host(self.chi2)
        beta = self.b["beta_host"]
        order = np.arange(self.nrep)
        start = self.rng.integers(0, 2)
        nsw = 0
        rates = np.full(self.nrep - 1, np.nan)
        for i in range(start, self.nrep - 1, 2):
            d = (beta[i] - beta[i + 1]) * (c2[order[i]] - c2[order[i + 1]]) * self.nfit
            ok = d >= 0 or self.rng.random() < np.exp(max(d, -60.0))
            rates[i] = 1.0 if ok else 0.0
            self.exch_attempts[i] += 1
            if ok:
                order[i], order[i + 1] = order[i + 1], order[i]
                nsw += 1
                self.exch_accepted[i] += 1
        if nsw:
            self.lad.apply_exchange(0, order)
        if return_rates:
            filled = np.where(np.isnan(rates),
                              np.nanmean(rates) if np.any(~np.isnan(rates)) else 0.3, rates)
            return nsw, filled
        return nsw

    def adapt(self, window_acc, window_exch):
        """Retune the displacement step and the ladder (method_a_rmc.py:376-398)."""
        if window_acc is not None and window_acc > 0:
            self.disp_sigma *= float(np.clip((window_acc / self.target_accept) ** 0.35, 0.7, 1.4))
            self.disp_sigma = float(np.clip(self.disp_sigma, 1e-4, 0.15))
            self.lad.set_field(0, "disp_sigma", self.disp_sigma)
        if window_exch is None or self.nrep < 4:
            return
        b = np.log(self.b["beta_host"])
        gaps = np.diff(b)
        rate = np.clip(window_exch, 0.02, 0.98)
        scale = (rate / max(rate.mean(), 1e-6)) ** 0.5
        gaps = gaps * scale
        gaps *= (b[-1] - b[0]) / gaps.sum()
        beta = np.exp(np.concatenate([[b[0]], b[0] + np.cumsum(gaps)]))
        self.b["beta_host"] = beta
        self.b["beta"].copy_(N.to_dev(beta))

    # ------------------------------------------------------------- loop
    def run(self, nsteps, exchange_every=25, log_every=500, callback=None):
        """Run the chain (method_a_rmc.py:401-455). Steps between two host
        events (exchange, adaptation, collection, log) go in one launch."""
        import torch
        hist = []
        acc_run = torch.zeros((), dtype=torch.float64, device="cuda")
        self._ensure_uniforms(self._stepc + nsteps)
        t0 = time.time()
        win_acc, win_exch = [], []

        def next_mult(it, every):
            return (it // every + 1) * every

        it = 0
        while it < nsteps:
            nxt = min(nsteps, it + MAX_BLOCK)
            for every in (exchange_every, self.adapt_every, log_every):
                if every:
                    nxt = min(nxt, next_mult(it, every))
            if it == 0:
                nxt = min(nxt, 1)
            if self.collect_after is not None:
                t = max(next_mult(it, self.collect_every), 0)
                while t - 1 < self.collect_after:
                    t += self.collect_every
                nxt = min(nxt, t)
            n = nxt - it
            flags = self.steps(n).double()
            per_step = flags.mean(dim=1)
            acc_run += per_step.sum()
            if self.adapt_every:
                win_acc.extend(per_step.unbind(0))
            it = nxt
            if exchange_every and it % exchange_every == 0:
                if self.reproduce:
                    _, per_pair = self.replica_exchange(return_rates=True)
                    if self.adapt_every:
                        win_exch.append(per_pair)
                else:
                    self.lad.exchange_device()
            if self.adapt_every and it % self.adapt_every == 0:
                wa = float(torch.stack(win_acc).mean()) if win_acc else None
                we = np.mean(win_exch, axis=0) if win_exch else None
                self.adapt(wa, we)
                win_acc, win_exch = [], []
            if (self.collect_after is not None and it - 1 >= self.collect_after
                    and it % self.collect_every == 0):
                self._collect()
            if it % log_every == 0 or it == 1:
                best = float(self.best_chi2.min())
                hist.append((it, best, float(acc_run) / it, time.time() - t0))
                if callback:
                    callback(it, best, hist[-1][2])
        if not self.reproduce:
            att = _host(self.b["exch_att"])[:self.nrep - 1]
            acc_ = _host(self.b["exch_acc"])[:self.nrep - 1]
            self.exch_attempts += att
            self.exch_accepted += acc_
            self.b["exch_att"].zero_()
            self.b["exch_acc"].zero_()
        self.lad.refresh_chi2()
        torch.cuda.synchronize()
        bsp, bpos, _ = self.best()
        chk = self.fm.chi_full(N.to_dev(bpos[None]), N.to_dev(bsp[None].astype(np.int32)),
                               precision=FP64)
        if self.ms is not None:
            chk = chk + self.ms.full(N.to_dev(bsp[None].astype(np.int32)))
        cnt = N.to_dev(np.array([[(bsp == s).sum() for s in range(self.nsp)]], np.float64))
        chi_in = chk.expand(self.lad.nslots, -1, -1).contiguous()
        cnt_in = cnt.expand(self.lad.nslots, -1).contiguous()
        self.best_verified = float(self.lad.eval_chi2(chi_in, cnt_in)[0])
        self.walltime = time.time() - t0
        self.history = hist
        with np.errstate(invalid="ignore", divide="ignore"):
            self.exchange_rate = np.where(self.exch_attempts > 0,
                                          self.exch_accepted / np.maximum(self.exch_attempts, 1),
                                          np.nan)
        if self.lad.device_error():
            raise N.ChxError(f"device error word {self.lad.device_error()} set during the run")
        return hist

    def collect_rungs(self):
        beta = self.b["beta_host"]
        k = min(self.n_collect, self.nrep)
        if self.collect_beta is None:
            return np.argsort(beta)[::-1][:k]
        return np.argsort(np.abs(np.log(beta) - np.log(self.collect_beta)))[:k]

    def _collect(self):
        idx = self.collect_rungs()
        sp = _host(self.species)[idx]
        c2 = _host(self.chi2)[idx]
        for a, b in zip(sp, c2):
            self.samples.append((a.astype(np.int32), float(b)))

    def posterior_wc(self, shell_r, i_idx, j_idx, shift, cell, nsp=None, tol=0.15):
        from .lattice import warren_cowley
        if not self.samples:
            raise RuntimeError("no samples collected; set collect_after in the constructor")
        n = nsp if nsp is not None else self.nsp
        arr = np.array([warren_cowley(sp, i_idx, j_idx, shift, cell, shell_r, tol=tol,
                                      nsp=n)[np.triu_indices(n)] for sp, _ in self.samples])
        return arr.mean(0), arr.std(0), len(arr)

    def best(self):
        bc = _host(self.b["best_chi2"])
        s = int(bc.argmin())
        return (_host(self.b["best_sp"][s]).astype(np.int32), _host(self.b["best_pos"][s]),
                float(bc[s]))


class BatchedSampler:
    """Many independent ladders in one launch per step, replayed as CUDA
    graphs (one graph = `exchange_every` steps + a device replica exchange),
    with FP64 re-anchoring of the running chi every `reanchor_every`
    accepted moves. By default (`device_reanchor`) the re-anchoring is part of
    every exchange period's graph: the device re-anchors the slots whose
    counter reached the threshold (at most `reanchor_cap` per period, the
    rest a period later), with no host round trip; otherwise the host checks
    the counters every `check_every` blocks.

    The step kernel is compiled per species count, so a batch that mixes
    binaries and ternaries is held as one group of ladders per count (in order
    of first appearance). Each exchange period launches every group's step
    and exchange on a stream of its own, forked from and joined back to the
    caller's stream, so the groups run side by side on the GPU and the whole
    period is still one graph replay. Ladder indices are global (the order of
    `specs`)."""

    def __init__(self, specs, precision=FP32C, exchange_every=25, use_table=True,
                 reanchor_every=1000, check_every=40, threads=256, min_blocks=3,
                 device_reanchor=True, reanchor_cap=8):
        import torch
        self.torch = torch
        specs = list(specs)
        counts = []
        for s in specs:
            if int(s.fm.nsp) not in counts:
                counts.append(int(s.fm.nsp))
        self.groups, self.where = [], [None] * len(specs)
        for g, nsp in enumerate(counts):
            idx = [i for i, s in enumerate(specs) if int(s.fm.nsp) == nsp]
            self.groups.append(Ladders([specs[i] for i in idx], precision=precision,
                                       use_table=use_table, threads=threads,
                                       min_blocks=min_blocks))
            for q, i in enumerate(idx):
                self.where[i] = (g, q)
        self._streams = None
        self.tuning = None
        self.exchange_every = int(exchange_every)
        self.reanchor_every = int(reanchor_every)
        self.check_every = int(check_every)
        self.device_reanchor = bool(device_reanchor) and self.reanchor_every > 0
        for lad in self.groups:     # slots re-anchored per period at most
            lad.reanchor_cap = int(reanchor_cap)
        self.graph = None
        self.blocks = 0
        self.host_reanchors = 0
        self.steps = 0

    @property
    def lad(self):
        """The Ladders of a batch with one species count."""
        if len(self.groups) != 1:
            raise ValueError("a batch of mixed species counts has one Ladders per count: "
                             "use .groups or .ladder(li)")
        return self.groups[0]

    def ladder(self, li):
        """(Ladders, index within it) of global ladder li."""
        g, q = self.where[li]
        return self.groups[g], q

    @property
    def nladders(self):
        return len(self.where)

    @property
    def nslots(self):
        return sum(g.nslots for g in self.groups)

    def init_state(self, species0, pos0):
        """species0 / pos0: one array per ladder (or one shared by all, then
        copied to the device once)."""
        from .forward import _dev
        torch = self.torch
        if not isinstance(species0, (list, tuple)):
            species0 = _dev(species0, torch.int32)
        if not isinstance(pos0, (list, tuple)):
            pos0 = _dev(pos0, torch.float64)
        for li in range(self.nladders):
            sp = species0[li] if isinstance(species0, (list, tuple)) else species0
            ps = pos0[li] if isinstance(pos0, (list, tuple)) else pos0
            lad, q = self.ladder(li)
            lad.init_state(q, sp, ps, defer=True)
        for lad in self.groups:
            lad.anchor_pending()
            lad.refresh_chi2(reset_best=True)

    def autotune(self, reps=3, path=None):
        """Measure the step kernel's launch shapes on this problem (real
        steps of the chains) and keep the fastest (chimera_b200.autotune),
        per group; the result of a one-group batch, else the list."""
        from .autotune import tune
        self.tuning = [tune(lad, nsteps=self.exchange_every, reps=reps, path=path)
                       for lad in self.groups]
        self.steps += self.exchange_every * (reps + 1) * 3
        return self.tuning[0] if len(self.groups) == 1 else self.tuning

    def device_error(self):
        """Error words of the groups OR-ed together (0 = none)."""
        e = 0
        for lad in self.groups:
            e |= lad.device_error()
        return e

    @property
    def reanchors(self):
        """Re-anchorings so far: slots re-anchored in the graph (device
        counters) plus host-side re-anchor launches."""
        return sum(lad.slot_reanchors() for lad in self.groups) + self.host_reanchors

    def _period(self, lad):
        lad.step(self.exchange_every)
        lad.exchange_device()
        if self.device_reanchor:
            lad.reanchor_due(self.reanchor_every)

    def block(self):
        """One exchange period: exchange_every steps in one launch, then the
        device exchange and the due re-anchorings (per group, the groups on
        parallel streams)."""
        if len(self.groups) == 1:
            self._period(self.groups[0])
            return
        torch = self.torch
        if self._streams is None:
            self._streams = [torch.cuda.Stream() for _ in self.groups]
        cur = torch.cuda.current_stream()
        for lad, st in zip(self.groups, self._streams):
            st.wait_stream(cur)
            with torch.cuda.stream(st):
                self._period(lad)
        for st in self._streams:
            cur.wait_stream(st)

    def capture(self):
        torch = self.torch
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.block()                      # sets kernel attributes before capture
        torch.cuda.current_stream().wait_stream(side)
        self.blocks += 1
        self.steps += self.exchange_every
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.block()
        self.graph = g
        return g

    def run_blocks(self, nblocks):
        if self.graph is None:
            self.capture()
        for _ in range(nblocks):
            self.graph.replay()
            self.blocks += 1
            self.steps += self.exchange_every
            if (self.collect_from is not None and self.blocks >= self.collect_from
                    and self.blocks % self.collect_every_blocks == 0):
                self.collect()
            if self.blocks % self.check_every == 0:
                if self.reanchor_every and not self.device_reanchor:
                    for lad in self.groups:
                        due = lad.accepted_since_anchor() >= self.reanchor_every
                        if bool(due.any()):
                            lad.reanchor(due)
                            self.host_reanchors += 1
                if self.surrogate is not None:
                    self._check_screen()

    # ------------------------------------------------- delayed acceptance
    surrogate = None
    da_max_err = 0.8        # screening error above which a ladder stops screening
    fallbacks = 0

    def learn(self, blocks=40, epochs=4, H=256, lr=1e-3, seed=0, batch=4096, cap=None):
        """Log the swaps of `blocks` exchange periods of plain steps, train
        surrogates on them (chimera_b200.surrogate) with one input row per
        chain (ladder and rung), and switch every ladder to delayed
        acceptance. A surrogate's input is the species around the swapped
        pair, so ladders share one when they have the same species count and
        feature width (lattices with the same first-shell coordination); a
        batch of several lattices or species counts trains one per class.
        Returns the training report (a list, one per class, when there are
        several)."""
        from .surrogate import SwapSurrogate
        for lad in self.groups:
            lad.enable_log(int(cap or self.exchange_every * blocks *
                               max(s.nrep for s in lad.specs)))
        self.graph = None
        self.run_blocks(blocks)
        old = getattr(self, "surrogates", None) or {}
        self.surrogates, reports = {}, []
        for g, lad in enumerate(self.groups):
            classes = {}
            for li in range(lad.nladders):
                lad.feature_table(li)
                classes.setdefault(int(lad.host[li].feat_D), []).append(li)
            for D, lis in classes.items():
                codes, lnb, y, chain, _ = lad.swap_log(ladders=lis, extra=True)
                sur = old.get((g, D))
                if sur is None or sur.H != H or sur.nchain != lad.nslots:
                    sur = SwapSurrogate(lad.nsp, D, H=H, nchain=lad.nslots, seed=seed)
                reports.append(sur.fit(codes, lnb, y, chain=chain, epochs=epochs, lr=lr,
                                       seed=seed, batch=batch))
                lad.attach_surrogate(sur, ladders=lis)
                self.surrogates[(g, D)] = sur
            lad.disable_log()
            lad.da_stats(reset=True)
        self.surrogate = next(iter(self.surrogates.values()))
        self.graph = None
        self.train_report = reports[0] if len(reports) == 1 else reports
        return self.train_report

    def _check_screen(self):
        """Ladders whose screening error since the last check exceeds
        da_max_err go back to plain steps. The screening error is the mean
        stage-2 rejection probability of the moves the screen let through,
        1 - mean min(1, exp(-beta nfit (d - d^))): 0 for an exact screen,
        the plain rejection rate for a screen that passes everything, the
        share of exact evaluations the screen could have saved.
        `last_screen` keeps the (nladders, 4) statistics in ladder order."""
        out = np.zeros((self.nladders, 4))
        for lad in self.groups:
            st = lad.da_stats(reset=True)
            on = lad.screening_on()
            for li in range(lad.nladders):
                if on[li] and st[li, 1] > 0:
                    err = 1.0 - st[li, 3] / st[li, 1]
                    if err > self.da_max_err:
                        lad.set_screening(li, False)
                        self.fallbacks += 1
            for gi, (g, q) in enumerate(self.where):
                if self.groups[g] is lad:
                    out[gi] = st[q]
        self.last_screen = out

    # ------------------------------------------------- posterior samples
    collect_from = None      # first exchange period (count) at which samples are taken

    def enable_collect(self, from_block, every_blocks=2, collect_beta=0.5, n_collect=4):
        """Posterior samples the way the reference's fit loop takes them
        (fitrun.py:307-333 with method_a_rmc.py:404-431, 458-491): from
        exchange period `from_block` on, every `every_blocks` periods (the
        reference's 50 steps are 2 periods of 25), the configurations of the
        n_collect rungs whose beta is nearest collect_beta in log spacing are
        reduced on the device to their first-shell pair-type counts
        (chx_pair_counts); `posterior_wc` turns them into Warren-Cowley
        parameters."""
        self.collect_from, self.collect_every_blocks = int(from_block), int(every_blocks)
        self.collect_beta, self.n_collect = float(collect_beta), int(n_collect)
        self._samples = [[] for _ in range(self.nladders)]
        self._shell_pairs = {}

    def _first_shell(self, fm):
        key = id(fm)
        if key not in self._shell_pairs:
            sel = np.asarray(fm.shell) == 0
            self._shell_pairs[key] = (N.to_dev(np.ascontiguousarray(fm.i_idx[sel], np.int32)),
                                      N.to_dev(np.ascontiguousarray(fm.j_idx[sel], np.int32)),
                                      int(sel.sum()))
        return self._shell_pairs[key]

    def collect(self):
        """Take one posterior sample set now (device work, no host sync)."""
        torch = self.torch
        for li in range(self.nladders):
            lad, q = self.ladder(li)
            b, spec = lad.bufs[q], lad.specs[q]
            beta = b["beta_host"]
            k = min(self.n_collect, spec.nrep)
            rungs = np.argsort(np.abs(np.log(beta) - np.log(self.collect_beta)))[:k]
            if "_collect_rungs" not in b:
                b["_collect_rungs"] = N.to_dev(np.ascontiguousarray(rungs, np.int64))
            rt = b["_collect_rungs"]
            sp = b["species"].index_select(0, b["slot_of"].index_select(0, rt).long()).contiguous()
            pi, pj, npair = self._first_shell(spec.fm)
            cnt = torch.empty((k, lad.nsp * lad.nsp), dtype=torch.int32, device="cuda")
            N.call("chx_pair_counts", N.ptr(sp), k, spec.fm.natoms, N.ptr(pi), N.ptr(pj), npair,
                   lad.nsp, N.ptr(cnt), N.ptr(lad.err), N.stream())
            self._samples[li].append((self.blocks, cnt))

    def posterior_wc(self, li, composition=None, from_block=None):
        """(mean, sd, n) of ladder li's first-shell Warren-Cowley vector (the
        upper triangle, lattice.wc_vector order) over its collected samples
        (method_a_rmc.py:477-491), those taken at or after exchange period
        from_block if given. composition: the species fractions (default the
        ladder's own, constant under swaps)."""
        lad, q = self.ladder(li)
        nsp = lad.nsp
        sel = [c for blk, c in self._samples[li] if from_block is None or blk >= from_block]
        if not sel:
            raise RuntimeError("no posterior samples: enable_collect before running")
        n = torch_cat_host(sel).reshape(-1, nsp, nsp).astype(np.float64)
        if composition is None:
            composition = _host(lad.bufs[q]["count"][0]) / lad.specs[q].fm.natoms
        c = np.asarray(composition, np.float64)
        tot = n.sum(2, keepdims=True)
        alpha = 1.0 - np.divide(n, np.maximum(tot, 1.0)) / c[None, None, :]
        alpha[np.broadcast_to(tot == 0, alpha.shape)] = 0.0
        iu = np.triu_indices(nsp)
        v = alpha[:, iu[0], iu[1]]
        return v.mean(0), v.std(0), v.shape[0]

    def best(self, li):
        lad, q = self.ladder(li)
        b = lad.bufs[q]
        bc = _host(b["best_chi2"])
        s = int(bc.argmin())
        return _host(b["best_sp"][s]).astype(np.int32), float(bc[s])

    def accept_rate(self):
        return sum(int(b["n_acc"].sum()) for lad in self.groups for b in lad.bufs)
