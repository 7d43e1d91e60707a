"""Global calibration in pair-count space with the population on the device.

The reference's calibration (chimera/calibrate.py:273-590) runs scipy's
differential evolution with one ShellModel.r_factor per population member
on the host. `Stage1` here is the reference's parameter vector of its global
search (calibrate.py:126-247: per-edge dE0, log sigma^2 scale, per-shell
log sigma^2 factors, free bond offsets, C3, C4, per-pair log widths, log MS
amplitude and c, per-edge MS amplitudes, k window, a0), mapped to rows of the
flat layout of chx_shell_rfactor; `de_stage1` runs the same differential
evolution with the whole population evaluated in one launch per generation
(scipy's `vectorized=True`, which implies deferred updating: every member of
a generation is scored before any replaces its parent).
"""
from __future__ import annotations

import numpy as np

from .shellmodel import ShellModel, as_kweights


def dr_from_free(x_free, comp):
    """Symmetric bond offsets from the free (a <= b) entries, the last
    diagonal fixed by sum_ab c_a c_b dr_ab = 0 (shellmodel.py:43-59)."""
    comp = np.asarray(comp, float)
    nsp = comp.size
    iu = np.triu_indices(nsp)
    w = np.array([comp[a] * comp[b] * (1.0 if a == b else 2.0) for a, b in zip(*iu)])
    x = np.zeros(w.size)
    x[:-1] = np.asarray(x_free, float)
    x[-1] = -(w[:-1] @ x[:-1]) / w[-1]
    dr = np.zeros((nsp, nsp))
    dr[iu] = x
    return dr + dr.T - np.diag(np.diag(dr))


def pair_log_from_free(x_free, comp):
    """Symmetric positive multipliers with composition-weighted geometric
    mean 1 from the free (a <= b) log entries (shellmodel.py:62-82)."""
    comp = np.asarray(comp, float)
    nsp = comp.size
    iu = np.triu_indices(nsp)
    w = np.array([comp[a] * comp[b] * (1.0 if a == b else 2.0) for a, b in zip(*iu)])
    u = np.zeros(w.size)
    u[:-1] = np.asarray(x_free, float)
    u[-1] = -(w[:-1] @ u[:-1]) / w[-1]
    U = np.zeros((nsp, nsp))
    U[iu] = u
    return np.exp(U + U.T - np.diag(np.diag(U)))


class Stage1:
    """Search vector <-> ShellModel parameters (names, bounds, unpack) of the
    reference's global stage, for the same flags."""

    def __init__(self, sm: ShellModel, comp, ms=True, free_window=True, free_dr=True,
                 free_c3=True, free_shell_sigma=True, dE0_bounds=None, dE0_start=0.0,
                 window_bounds=((2.5, 4.0), (11.0, 15.0)), with_sigma=True, free_a0=False,
                 a0_bounds=None, free_c4=False, free_sigma_pair=False, free_ms_edge=False,
                 elements=None):
        self.sm, self.comp = sm, np.asarray(comp, float)
        self.nsp = int(self.comp.size)
        els = tuple(elements) if elements else tuple(f"e{i}" for i in range(self.nsp))
        pairs = [f"{els[a]}{els[b]}" for a in range(self.nsp) for b in range(a, self.nsp)]
        if a0_bounds is None:
            a0_bounds = (sm.a0_ref * 0.953, sm.a0_ref * 1.0236)
        self.names, self.bounds = [], []

        def add(name, lo, hi):
            self.names.append(name)
            self.bounds.append((float(lo), float(hi)))

        self.dE0_start = float(dE0_start)
        if dE0_bounds is None:
            dE0_bounds = (self.dE0_start - 17.0, self.dE0_start + 23.0)
        for e in range(self.nsp):
            add(f"dE0_{els[e]}", *dE0_bounds)
        self.with_sigma = bool(with_sigma)
        if with_sigma:
            add("log_sigma", np.log(0.5), np.log(6.0))
        self.nsss = sm.nshell - 1 if free_shell_sigma else 0
        for s in range(1, sm.nshell) if free_shell_sigma else ():
            add(f"log_sigma_shell{s + 1}", np.log(0.4), np.log(2.5))
        self.ndr = len(pairs) - 1 if free_dr else 0
        for lab in pairs[:self.ndr]:
            add(f"dr_{lab}", -0.06, 0.06)
        self.c3 = bool(free_c3)
        if free_c3:
            add("c3", -6e-4, 6e-4)
        self.c4 = bool(free_c4)
        if free_c4:
            add("c4", -3e-5, 3e-5)
        self.nsp_pair = (len(pairs) - 1) if free_sigma_pair else 0
        for lab in pairs[:self.nsp_pair]:
            add(f"logs2_{lab}", -0.7, 0.7)
        self.ms = bool(ms)
        if ms:
            add("log_ms_amp", np.log(0.3), np.log(2.5))
            add("log_ms_c", np.log(0.4), np.log(3.0))
        self.ms_edge = bool(ms and free_ms_edge)
        for e in range(self.nsp - 1) if self.ms_edge else ():
            add(f"log_ms_{els[e]}", -0.5, 0.5)
        self.window = bool(free_window)
        if free_window:
            add("kmin", *window_bounds[0])
            add("kmax", *window_bounds[1])
        self.free_a0 = bool(free_a0)
        if free_a0:
            add("a0", *a0_bounds)

    def unpack(self, x):
        """Parameter dict of one search vector (calibrate.py:195-225)."""
        x = np.asarray(x, float)
        i = 0
        p = dict(dE0=x[i:i + self.nsp].copy())
        i += self.nsp
        if self.with_sigma:
            p["sigma_scale"] = float(np.exp(x[i]))
            i += 1
        if self.nsss:
            sss = np.ones(self.sm.nshell)
            sss[1:] = np.exp(x[i:i + self.nsss])
            p["sigma_shell_scale"] = sss
            i += self.nsss
        if self.ndr:
            p["dr"] = dr_from_free(x[i:i + self.ndr], self.comp)
            i += self.ndr
        if self.c3:
            p["c3"] = [float(x[i])]
            i += 1
        if self.c4:
            p["c4"] = [float(x[i])]
            i += 1
        if self.nsp_pair:
            p["sigma_pair"] = pair_log_from_free(x[i:i + self.nsp_pair], self.comp)
            i += self.nsp_pair
        if self.ms:
            p["ms_amp"] = float(np.exp(x[i]))
            p["ms_c"] = float(np.exp(x[i + 1]))
            i += 2
        if self.ms_edge:
            u = np.zeros(self.nsp)
            u[:self.nsp - 1] = x[i:i + self.nsp - 1]
            u[-1] = -u[:-1].sum()
            p["ms_amp_edge"] = np.exp(u)
            i += self.nsp - 1
        if self.window:
            p["kmin"] = float(x[i])
            p["kmax"] = float(x[i + 1])
            i += 2
        if self.free_a0:
            p["a0"] = float(x[i])
            i += 1
        return p

    def x0(self):
        """The reference's default starting vector (calibrate.py:227-247)."""
        defaults = dict(log_sigma=np.log(3.0), log_ms_amp=0.0, log_ms_c=np.log(1.3),
                        kmin=3.0, kmax=13.0, a0=self.sm.a0_ref)
        return np.array([self.dE0_start if n.startswith("dE0") else defaults.get(n, 0.0)
                         for n in self.names])

    def rows(self, X, a0=None):
        """Flat parameter rows of the search vectors X (P, ndim), one
        `unpack` and set_params per vector (the reference's path)."""
        dicts = []
        for x in np.atleast_2d(X):
            p = self.unpack(x)
            if a0 is not None:
                p.setdefault("a0", a0)
            dicts.append(p)
        return self.sm.flat_rows(dicts)

    def rows_fast(self, X, a0=None):
        """The rows of `rows`, for a whole population at once: every block of
        the vector maps to the flat layout linearly (bond offsets and pair-
        width logs through their free-entry bases) or through exp."""
        sm, nsp, nsh = self.sm, self.nsp, self.sm.nshell
        X = np.atleast_2d(np.asarray(X, float))
        P = X.shape[0]
        sl = sm._slices()
        out = np.tile(sm.flat(), (P, 1))
        if a0 is not None and not self.free_a0:
            out[:, sl["a0"]] = a0
        i = 0
        out[:, sl["dE0"]] = X[:, i:i + nsp]
        i += nsp
        if self.with_sigma:
            out[:, sl["sigma_scale"]] = np.exp(X[:, i:i + 1])
            i += 1
        if self.nsss:
            sss = np.ones((P, nsh))
            sss[:, 1:] = np.exp(X[:, i:i + self.nsss])
            out[:, sl["sigma_shell_scale"]] = sss
            i += self.nsss
        if self.ndr:
            basis = np.array([dr_from_free(np.eye(self.ndr)[q], self.comp).ravel()
                              for q in range(self.ndr)])
            out[:, sl["dr"]] = X[:, i:i + self.ndr] @ basis
            i += self.ndr
        if self.c3:
            c = np.zeros((P, nsh))
            c[:, 0] = X[:, i]
            out[:, sl["c3"]] = c
            i += 1
        if self.c4:
            c = np.zeros((P, nsh))
            c[:, 0] = X[:, i]
            out[:, sl["c4"]] = c
            i += 1
        if self.nsp_pair:
            basis = np.array([np.log(pair_log_from_free(np.eye(self.nsp_pair)[q],
                                                        self.comp)).ravel()
                              for q in range(self.nsp_pair)])
            out[:, sl["sigma_pair"]] = np.exp(X[:, i:i + self.nsp_pair] @ basis)
            i += self.nsp_pair
        if self.ms:
            out[:, sl["ms_amp"]] = np.exp(X[:, i:i + 1])
            out[:, sl["ms_c"]] = np.exp(X[:, i + 1:i + 2])
            i += 2
        if self.ms_edge:
            u = np.zeros((P, nsp))
            u[:, :nsp - 1] = X[:, i:i + nsp - 1]
            u[:, -1] = -u[:, :-1].sum(1)
            out[:, sl["ms_amp_edge"]] = np.exp(u)
            i += nsp - 1
        if self.window:
            out[:, sl["kmin"]] = X[:, i:i + 1]
            out[:, sl["kmax"]] = X[:, i + 1:i + 2]
            i += 2
        if self.free_a0:
            out[:, sl["a0"]] = X[:, i:i + 1]
            i += 1
        return out


def de_stage1(sm: ShellModel, Nc, data, mask, idx, stage: Stage1, kweight=None, a0=None,
              maxiter=120, popsize=12, seed=0, tol=1e-8, polish=True, x0=None):
    """Differential evolution of the stage's vector against `data`, every
    generation one chx_shell_rfactor launch (scipy vectorized mode).
    Returns (scipy OptimizeResult, number of members evaluated)."""
    from scipy.optimize import differential_evolution
    if kweight is not None:
        sm.set_params(kweight=as_kweights(kweight))
    calls = [0]

    def score(xT):
        X = np.asarray(xT, float)
        X = X[:, None] if X.ndim == 1 else X
        rows = stage.rows_fast(X.T, a0=a0)
        calls[0] += rows.shape[0]
        rf, _ = sm.r_factor_batch(Nc, data, mask, idx, rows)
        rf = np.where(np.isfinite(rf), rf, np.inf)
        return rf if np.ndim(xT) > 1 else float(rf[0])

    res = differential_evolution(score, stage.bounds, maxiter=maxiter, popsize=popsize,
                                 seed=seed, tol=tol, polish=polish, vectorized=True,
                                 updating="deferred",
                                 x0=stage.x0() if x0 is None else x0)
    return res, calls[0]
