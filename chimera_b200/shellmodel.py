"""Pair-count (shell) calibration objective on the device (chimera/shellmodel.py).

On ideal sites chi depends on the configuration only through the ordered
pair counts N[a, b, s], and the calibration (chimera/calibrate.py) searches
the model's parameters - lattice constant, E0 shifts, k window, sigma^2
scales, bond offsets, cumulants, MS amplitude - with differential evolution,
one `ShellModel.r_factor` per population member on the host. Here the whole
population is one launch of `chx_shell_rfactor`: per member the basis at its
parameters, the contraction with N, the averaged MS term, each channel's
resampling onto the member's own k axis and window, the transform on the
fitted R points, the profiled per-edge amplitudes and the R-factor.

`ShellModel` keeps the reference class's parameter set and defaults
(shellmodel.py:101-150, set_params :231-262), its pair-count helpers
(counts_of, absorber_counts, random_counts, alpha :375-408) and r_factor
(:427-440, evaluated on the device), and adds `r_factor_batch` over rows of
the flat parameter layout of chx_shell_rfactor (`flat`, `PARAM_ORDER`). The
physical per-pair tables of `set_physics` are not carried.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

ETOK = 0.2624682843          # k^2 (A^-2) per eV of E0 shift (chimera/model.py:94)
PARAM_ORDER = ("a0", "sigma_scale", "ms_amp", "ms_c", "kmin", "kmax", "dE0",
               "sigma_shell_scale", "dr", "c3", "c4", "sigma_pair", "ms_amp_edge")


def as_kweights(kw):
    kw = tuple(int(x) for x in np.atleast_1d(kw))
    return kw


class ShellModel:
    """chi from pair counts and the calibration R-factor, on the device."""

    def __init__(self, k_phys, tables, shells_ref, shell_mult, sigma2_shell_ref, natoms,
                 a0_ref, ms_paths=None, s02=1.0, dk_win=1.0, pairs=None, composition=None,
                 elements=None, nfft=2048, dk=0.05, etok=ETOK):
        self.k = np.asarray(k_phys, float)
        _, f, delta, lam = tables.as_float64() if hasattr(tables, "as_float64") else tables
        self.f = np.asarray(f, float)
        self.nsp = int(self.f.shape[0])
        self.delta = np.asarray(delta, float).reshape(self.nsp * self.nsp, -1)
        self.lam = np.asarray(lam, float)
        comp = (np.ones(self.nsp) / self.nsp if composition is None
                else np.asarray(composition, float))
        self.composition = tuple(float(x) for x in comp / comp.sum())
        self.elements = tuple(elements) if elements is not None else None
        self.shells_ref = np.asarray(shells_ref, float)
        self.nshell = int(self.shells_ref.size)
        self.z = np.asarray(shell_mult, float)
        self.sigma2_shell_ref = np.asarray(sigma2_shell_ref, float)
        self.natoms = int(natoms)
        self.a0_ref = float(a0_ref)
        self.s02, self.dk_win, self.nfft, self.dk, self.etok = (float(s02), float(dk_win),
                                                                int(nfft), float(dk), float(etok))
        self.pairs = pairs
        self.ms = self._ms_arrays(ms_paths)
        self.p = dict(a0=self.a0_ref, dE0=np.zeros(self.nsp), kmin=3.0, kmax=13.0,
                      kweight=(3,), sigma_scale=1.0, sigma_shell_scale=np.ones(self.nshell),
                      dr=np.zeros((self.nsp, self.nsp)), c3=np.zeros(self.nshell),
                      ms_amp=1.0, ms_c=1.3, c4=np.zeros(self.nshell),
                      sigma_pair=np.ones((self.nsp, self.nsp)), ms_amp_edge=np.ones(self.nsp))
        self._dev = None
        self.nparam = int(N.lib().chx_shell_nparam(self.nsp, self.nshell))

    # --------------------------------------------------------- parameters
    def set_params(self, **kw):
        """The reference's set_params (shellmodel.py:231-262)."""
        for key, v in kw.items():
            if key not in self.p:
                raise KeyError(f"unknown parameter {key!r}")
            if v is None:
                continue
            if key == "dE0":
                v = np.asarray(v, float) * np.ones(self.nsp)
            elif key == "sigma_shell_scale":
                v = np.asarray(v, float).ravel()
                assert v.size == self.nshell, f"need {self.nshell} per-shell factors"
            elif key in ("dr", "sigma_pair"):
                v = np.asarray(v, float).reshape(self.nsp, self.nsp)
            elif key in ("c3", "c4"):
                c = np.atleast_1d(np.asarray(v, float))
                v = np.zeros(self.nshell)
                v[:min(c.size, self.nshell)] = c[:self.nshell]
            elif key == "ms_amp_edge":
                v = np.asarray(v, float).ravel() * np.ones(self.nsp)
            elif key == "kweight":
                v = as_kweights(v)
            elif key in ("kmin", "kmax"):
                v = float(np.atleast_1d(v)[0])
            else:
                v = float(v)
            self.p[key] = v
        return self

    def _slices(self):
        sizes = dict(a0=1, sigma_scale=1, ms_amp=1, ms_c=1, kmin=1, kmax=1, dE0=self.nsp,
                     sigma_shell_scale=self.nshell, dr=self.nsp ** 2, c3=self.nshell,
                     c4=self.nshell, sigma_pair=self.nsp ** 2, ms_amp_edge=self.nsp)
        out, o = {}, 0
        for k in PARAM_ORDER:
            out[k] = slice(o, o + sizes[k])
            o += sizes[k]
        return out

    def set_flat(self, row):
        """Set every parameter from one row of the flat layout."""
        sl = self._slices()
        row = np.asarray(row, float)
        assert row.size == self.nparam
        for k in PARAM_ORDER:
            v = row[sl[k]]
            if k in ("dr", "sigma_pair"):
                v = v.reshape(self.nsp, self.nsp)
            elif v.size == 1 and k not in ("dE0", "ms_amp_edge", "sigma_shell_scale", "c3", "c4"):
                v = float(v[0])
            self.p[k] = v.copy() if isinstance(v, np.ndarray) else v
        return self

    def flat(self, p=None):
        """One row of the flat layout: the current parameters, with the
        entries of the dict `p` (set_params conventions) overriding."""
        return self.flat_rows([p or {}])[0]

    def flat_rows(self, dicts):
        """(len(dicts), nparam) rows: the current parameters, each row with
        its dict's entries (set_params conventions) overriding."""
        sl = self._slices()
        base = np.concatenate([np.asarray(self.p[k], float).ravel() for k in PARAM_ORDER])
        out = np.tile(base, (len(dicts), 1))
        keep = {k: self.p[k] for k in PARAM_ORDER}
        for r, d in enumerate(dicts):
            if not d:
                continue
            self.set_params(**{k: v for k, v in d.items() if k != "kweight"})
            for k in d:
                if k in sl:
                    out[r, sl[k]] = np.asarray(self.p[k], float).ravel()
            self.p.update(keep)
        return out

    # ------------------------------------------------------ pair counts
    def counts_of(self, species):
        """Ordered pair counts N[a, b, s] of a configuration (:379-386)."""
        assert self.pairs is not None, "ShellModel built without pair lists"
        i, j, sh = self.pairs
        sp = np.asarray(species, int)
        Nc = np.zeros((self.nsp, self.nsp, self.nshell))
        np.add.at(Nc, (sp[i], sp[j], sh), 1.0)
        return Nc

    def absorber_counts(self, Nc):
        return np.asarray(Nc).sum(axis=(1, 2)) / self.z.sum()

    def random_counts(self, composition=None, counts=None):
        """Expected pair counts of a random alloy: N[a,b,s] = N_a z_s c_b."""
        if counts is None:
            comp = (np.asarray(self.composition, float) if composition is None
                    else np.asarray(composition, float))
            cnt = np.round(comp / comp.sum() * self.natoms).astype(int)
            cnt[-1] = self.natoms - cnt[:-1].sum()
        else:
            cnt = np.asarray(counts, int)
        c = cnt / cnt.sum()
        return cnt[:, None, None] * self.z[None, None, :] * c[None, :, None]

    def alpha(self, Nc, s=0):
        cnt = self.absorber_counts(Nc)
        c = cnt / cnt.sum()
        return 1.0 - np.asarray(Nc)[:, :, s] / np.maximum(cnt[:, None] * self.z[s] * c[None, :],
                                                          1e-30)

    # -------------------------------------------------------- device side
    @staticmethod
    def _ms_arrays(ms):
        """Flatten a prepared averaged-MS path set: the reference's MSPaths
        after `prepare` (elements, _prep[a] = (reff, deg, F, D, L), d_nn) or
        a dict with absorber, reff, deg, F, D, L, dnn."""
        if ms is None:
            return None
        if isinstance(ms, dict):
            return {k: np.asarray(v) for k, v in ms.items()}
        ab, R, G, F, D, L = [], [], [], [], [], []
        for e, a in enumerate(ms.elements):
            reff, deg, f, d, lam = ms._prep[a]
            ab.append(np.full(len(reff), e))
            R.append(reff); G.append(deg); F.append(f); D.append(d); L.append(lam)
        return dict(absorber=np.concatenate(ab), reff=np.concatenate(R), deg=np.concatenate(G),
                    F=np.vstack(F), D=np.vstack(D), L=np.vstack(L), dnn=float(ms.d_nn))

    def _fixed(self):
        if self._dev is None:
            d = {k: N.to_dev(np.ascontiguousarray(v, np.float64)) for k, v in
                 dict(k=self.k, f=self.f, delta=self.delta, lam=self.lam,
                      shells_ref=self.shells_ref, sigma2_ref=self.sigma2_shell_ref,
                      shell_mult=self.z).items()}
            if self.ms is not None:
                for k in ("reff", "deg", "F", "D", "L"):
                    d["ms_" + k] = N.to_dev(np.ascontiguousarray(self.ms[k], np.float64))
                d["ms_abs"] = N.to_dev(np.ascontiguousarray(self.ms["absorber"], np.int32))
            self._dev = d
        return self._dev

    def r_factor_batch(self, Nc, data, mask, idx, X, kweight=None, magnitude=None):
        """R-factor and per-edge amplitudes (P,), (P, nsp) of the pair counts
        Nc for every row of X (P, nparam) against `data` (nchan, nR) on the
        model R grid points idx, fitted over mask. magnitude: fit |chi(R)|
        (default: when data is real)."""
        rf, sc, _ = self._launch(Nc, data, mask, idx, X, kweight, magnitude)
        return rf, sc

    def residual_batch(self, Nc, data, mask, idx, X, sigma=None, profile=True, kweight=None,
                       magnitude=None):
        """Residuals (scale m - data) / sigma on the fitted points of every
        member, ordered as chimera/shellmodel.py:504-508 orders them (channel-
        major; the real parts, then the imaginary parts for complex data).
        Nc is one (nsp, nsp, nshell) array or one per member (P, ...)."""
        rf, sc, r = self._launch(Nc, data, mask, idx, X, kweight, magnitude, resid=True,
                                 sigma=sigma, profile=profile)
        cplx = np.iscomplexobj(data) if magnitude is None else not magnitude
        re, im = r[..., 0].reshape(len(r), -1), r[..., 1].reshape(len(r), -1)
        return np.concatenate([re, im], axis=1) if cplx else re

    def _launch(self, Nc, data, mask, idx, X, kweight=None, magnitude=None, resid=False,
                sigma=None, profile=True):
        import torch
        d = self._fixed()
        kw = as_kweights(self.p["kweight"] if kweight is None else kweight)
        data = np.asarray(data)
        mask = np.asarray(mask, bool)
        mag = (not np.iscomplexobj(data)) if magnitude is None else bool(magnitude)
        bins = np.asarray(idx)[mask].astype(np.int32)
        dm = data[:, mask]
        dd = np.stack([dm.real, dm.imag if np.iscomplexobj(dm) else np.zeros_like(dm.real)],
                      axis=-1).astype(np.float64)
        nchan = self.nsp * len(kw)
        assert dd.shape[0] == nchan, "data must have one row per (edge, k weight)"
        X = np.ascontiguousarray(np.atleast_2d(X), np.float64)
        assert X.shape[1] == self.nparam, f"need {self.nparam} parameters per row"
        P = X.shape[0]
        Nc = np.ascontiguousarray(Nc, np.float64)
        per_member = Nc.ndim == 4
        assert not per_member or Nc.shape[0] == P, "one pair-count array per member"
        t = dict(N=N.to_dev(Nc), kw=N.to_dev(np.array(kw, np.int32)), bins=N.to_dev(bins),
                 data=N.to_dev(np.ascontiguousarray(dd)), X=N.to_dev(X))
        rf = torch.empty(P, dtype=torch.float64, device="cuda")
        sc = torch.empty((P, self.nsp), dtype=torch.float64, device="cuda")
        S = N.Shell()
        S.nsp, S.nshell, S.nk, S.nkw, S.nbin, S.nfft = (self.nsp, self.nshell, self.k.size,
                                                        len(kw), bins.size, self.nfft)
        S.magnitude, S.profile = int(mag), int(bool(profile))
        S.a0_ref, S.s02, S.dk_win, S.dk, S.etok = (self.a0_ref, self.s02, self.dk_win, self.dk,
                                                   self.etok)
        S.k, S.f, S.delta, S.lam = (N.dptr(d["k"]), N.dptr(d["f"]), N.dptr(d["delta"]),
                                    N.dptr(d["lam"]))
        S.shells_ref, S.sigma2_ref, S.shell_mult = (N.dptr(d["shells_ref"]),
                                                    N.dptr(d["sigma2_ref"]),
                                                    N.dptr(d["shell_mult"]))
        if per_member:
            S.N_member = N.dptr(t["N"])
        else:
            S.N = N.dptr(t["N"])
        S.kweight, S.bins, S.data = N.dptr(t["kw"]), N.dptr(t["bins"]), N.dptr(t["data"])
        r = None
        if resid:
            r = torch.empty((P, nchan, bins.size, 2), dtype=torch.float64, device="cuda")
            S.resid = N.dptr(r)
            if sigma is not None:
                sg = np.asarray(sigma, float)
                if sg.ndim == 0:
                    sg = np.full((nchan, data.shape[1]), float(sg))
                elif sg.ndim == 1:                      # per channel (shellmodel.py:496-498)
                    sg = np.repeat(sg[:, None], data.shape[1], axis=1)
                sg = sg[:, mask]
                t["sigma"] = N.to_dev(np.ascontiguousarray(sg))
                S.sigma = N.dptr(t["sigma"])
        if self.ms is not None:
            S.npath, S.ms_dnn = int(self.ms["reff"].size), float(self.ms["dnn"])
            S.ms_abs, S.ms_reff, S.ms_deg = (N.dptr(d["ms_abs"]), N.dptr(d["ms_reff"]),
                                             N.dptr(d["ms_deg"]))
            S.ms_F, S.ms_D, S.ms_L = N.dptr(d["ms_F"]), N.dptr(d["ms_D"]), N.dptr(d["ms_L"])
        N.call("chx_shell_rfactor", C.byref(S), N.ptr(t["X"]), P, N.ptr(rf), N.ptr(sc),
               N.stream())
        return rf.cpu().numpy(), sc.cpu().numpy(), (None if r is None else r.cpu().numpy())

    def r_factor(self, Nc, data, mask, idx, return_scales=False):
        """The reference's r_factor (shellmodel.py:427-440) at the current
        parameters, on the device."""
        rf, sc = self.r_factor_batch(Nc, data, mask, idx, self.flat()[None])
        return (float(rf[0]), sc[0]) if return_scales else float(rf[0])


# ================================================================ Fisher bounds
# Prior widths, nuisance list and finite-difference steps of the reference's
# bound (chimera/shellmodel.py:444-446, 491-493), kept identical so that the
# bounds are the same numbers.
PRIOR_SD = dict(alpha=1.0, a0=0.02, sigma_scale=0.5, ms_amp=0.5, ms_c=0.5, c3=2e-4,
                dE0=5.0, dr=0.05)
NUISANCE_DEFAULT = ("a0", "sigma_scale", "ms_amp", "dE0", "dr", "c3")
STEPS = dict(a0=0.002, sigma_scale=0.05, ms_amp=0.05, ms_c=0.05, c3=2e-5, dE0=0.5, dr=0.005)


def sro_directions(nsp):
    """Independent short-range-order directions per shell: (a, b), a < b."""
    return [(a, b) for a in range(nsp) for b in range(a + 1, nsp)]


def dN_direction(nsp, nshell, s, a, b):
    """+1 on (a,b) and (b,a), -1 on (a,a) and (b,b) in shell s: a change of
    the pair counts that keeps every absorber's coordination."""
    d = np.zeros((nsp, nsp, nshell))
    d[a, b, s] += 1.0
    d[b, a, s] += 1.0
    d[a, a, s] -= 1.0
    d[b, b, s] -= 1.0
    return d


def crlb(model: ShellModel, Nc, data, sigma, mask, idx, shells=None, alpha_shell=0,
         nuisance=NUISANCE_DEFAULT, profile_scale=True, threshold=0.3, steps=None,
         prior_sd=None, whiten=None):
    """Cramer-Rao bounds on the shell-`alpha_shell` Warren-Cowley parameters
    (chimera/shellmodel.py:449-593): the Jacobian of the sigma-scaled
    residual along the SRO directions of every shell in `shells` and the
    nuisance parameters by central differences, all 2 x ncolumn perturbed
    models in one chx_shell_rfactor launch, then the FP64 Fisher matrix with
    a weak Gaussian prior, its inverse and the marginal widths on the host.
    Returns the reference's dictionary."""
    from .calibrate import dr_from_free
    nsp, nshell = model.nsp, model.nshell
    shells = list(range(nshell)) if shells is None else list(shells)
    Nc = np.asarray(Nc, float)
    cnt = model.absorber_counts(Nc)
    c = cnt / cnt.sum()
    iu = np.triu_indices(nsp)
    st = dict(STEPS)
    if steps:
        st.update(steps)
    pr = dict(PRIOR_SD)
    if prior_sd:
        pr.update(prior_sd)
    Ns, dicts, step_of, A, names, prec = [], [], [], [], [], []
    for s in shells:
        h = 0.02 * cnt.min() * model.z[s] * c.min()
        for a, b in sro_directions(nsp):
            d = dN_direction(nsp, nshell, s, a, b)
            Ns += [Nc + h * d, Nc - h * d]
            dicts += [{}, {}]
            step_of.append(h)
            names.append(f"sro_s{s + 1}_{a}{b}")
            dalpha = (model.alpha(Nc + h * d, s) - model.alpha(Nc, s)) / h
            A.append(dalpha[iu] if s == alpha_shell else np.zeros(len(iu[0])))
            prec.append((np.abs(dalpha).max() / pr["alpha"]) ** 2)
    nsro = len(names)
    saved = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in model.p.items()}

    def column(name, hi_, lo_, step):
        Ns.extend([Nc, Nc])
        dicts.extend([{name: hi_}, {name: lo_}])
        step_of.append(step)
        prec.append(1.0 / pr[name] ** 2)

    ndr_free = nsp * (nsp + 1) // 2 - 1
    for name in nuisance or ():
        v0 = saved[name]
        if name == "a0":
            column(name, v0 + st[name], v0 - st[name], st[name])
            names.append(name)
        elif name == "c3":
            hi_ = v0.copy()
            hi_[0] += st[name]
            lo_ = v0.copy()
            lo_[0] -= st[name]
            column(name, hi_, lo_, st[name])
            names.append(name)
        elif name == "dE0":
            for e in range(nsp):
                hi_ = v0.copy()
                hi_[e] += st[name]
                lo_ = v0.copy()
                lo_[e] -= st[name]
                column(name, hi_, lo_, st[name])
                names.append(f"dE0_{e}")
        elif name == "dr":
            for q in range(ndr_free):
                e_ = np.zeros(ndr_free)
                e_[q] = st[name]
                d = dr_from_free(e_, c)
                column(name, v0 + d, v0 - d, st[name])
                names.append(f"dr_{q}")
        else:
            column(name, v0 * np.exp(st[name]), v0 * np.exp(-st[name]), st[name])
            names.append(name)
    X = model.flat_rows(dicts)
    R = model.residual_batch(np.array(Ns), data, mask, idx, X, sigma=sigma,
                             profile=profile_scale)
    if whiten is not None:
        R = np.array([whiten(r) for r in R])
    J = ((R[0::2] - R[1::2]) / (2.0 * np.asarray(step_of))[:, None]).T
    F = J.T @ J
    cov = np.linalg.inv(F + np.diag(prec))
    A = np.array(A)
    cov_alpha = A.T @ cov[:nsro, :nsro] @ A
    sd = np.sqrt(np.maximum(np.diag(cov_alpha), 0.0))
    ev = np.linalg.eigvalsh(F[:nsro, :nsro])[::-1]
    with np.errstate(divide="ignore"):
        eig_sd = 1.0 / np.sqrt(np.maximum(ev, 1e-300))
    csd = np.sqrt(np.maximum(np.diag(cov), 0.0))
    nuis_sd = {}
    for j, name in enumerate(names[nsro:], start=nsro):
        key = name.split("_")[0] if name.startswith(("dE0_", "dr_")) else name
        nuis_sd.setdefault(key, []).append(float(csd[j]))
    dr_entry_sd = None
    if "dr" in nuis_sd:
        q = [j for j, n in enumerate(names) if n.startswith("dr_")]
        D = np.array([dr_from_free(np.eye(ndr_free)[i], c)[iu] for i in range(ndr_free)])
        dr_entry_sd = np.sqrt(np.maximum(np.einsum("ie,ij,je->e", D, cov[np.ix_(q, q)], D),
                                         0.0)).tolist()
    return dict(alpha_sd=sd.tolist(), determined=(sd < threshold).tolist(),
                threshold=threshold, prior_alpha_sd=pr["alpha"],
                shells=[int(s) + 1 for s in shells], nuisance=list(nuisance or ()),
                n_sro_directions=int(nsro), eig_sd=eig_sd.tolist(), columns=names,
                alpha_cov=cov_alpha.tolist(),
                nuisance_sd={k: (v[0] if len(v) == 1 else v) for k, v in nuis_sd.items()},
                dr_entry_sd=dr_entry_sd, n_models=len(Ns))
