"""k -> R transform with the reference's EXAFS conventions (exafs_gpu/fourier.py).

Set-up is the reference's, array for array (fourier.py:21-67): the uniform
grid k_n = n dk (n < nfft), the Hanning window of taper dk_win times k^w
(zeroed outside the model grid), linear resampling precomputed as index and
fraction, and norm dk / sqrt(pi). The transform sign is the reference code's,
e^{-2ikR} (numpy/cuFFT forward FFT, fourier.py:79), and the R grid is
m pi / (nfft dk).

Evaluation runs on the device only: the resample-window-FFT chain is linear,
so it is folded into one complex basis B (nk, nbins) and applied as a dense
contraction by `chx_ft_batch` (FP64 by default). Host NumPy input (the
reference's `xp=np` callers, chimera/chik.py:141-144) goes through the same
device path and comes back as NumPy.

The benchmark configurations also name a Kaiser window, which the reference
does not have; `kaiser_window` implements the Kaiser-Bessel taper of Kaiser &
Schafer (1980) on the same support as the Hanning window:
    w(k) = I0(beta * sqrt(1 - u^2)) / I0(beta),  u = (k - kc) / hw,
kc = (kmin + kmax) / 2, hw = (kmax - kmin + dk_win) / 2, zero for |u| > 1,
with shape parameter beta (default 4).
"""
from __future__ import annotations

import numpy as np

from . import _native as N

DK = 0.05
NFFT = 2048


def r_grid(nfft=NFFT, dk=DK):
    return np.arange(nfft // 2) * np.pi / (nfft * dk)


def hanning_window(k, kmin, kmax, dk_win=1.0):
    """Hanning window with sine tapers of width dk_win (fourier.py:25-33)."""
    w = np.zeros_like(k)
    w[(k >= kmin + dk_win / 2) & (k <= kmax - dk_win / 2)] = 1.0
    lo = (k > kmin - dk_win / 2) & (k < kmin + dk_win / 2)
    w[lo] = 0.5 * (1 + np.sin(np.pi * (k[lo] - kmin) / dk_win))
    hi = (k > kmax - dk_win / 2) & (k < kmax + dk_win / 2)
    w[hi] = 0.5 * (1 - np.sin(np.pi * (k[hi] - kmax) / dk_win))
    return w


def kaiser_window(k, kmin, kmax, dk_win=1.0, beta=4.0):
    """Kaiser-Bessel taper (see module docstring)."""
    kc = 0.5 * (kmin + kmax)
    hw = 0.5 * (kmax - kmin + dk_win)
    u = (np.asarray(k, float) - kc) / hw
    arg = np.clip(1.0 - u * u, 0.0, None)
    w = np.i0(beta * np.sqrt(arg)) / np.i0(beta)
    w[np.abs(u) > 1.0] = 0.0
    return w


class FourierTransform:
    """Resamples chi(k) onto the uniform grid and transforms to R space."""

    def __init__(self, k_model, kmin=3.0, kmax=14.0, kweight=2, dk_win=1.0, nfft=NFFT,
                 dk=DK, xp=None, window="hanning", beta=4.0):
        self.xp = xp
        self.nfft, self.dk, self.kweight = int(nfft), float(dk), kweight
        self.k_model = np.asarray(k_model, float)
        self.k_uniform = np.arange(nfft) * dk
        self.kmin, self.kmax = kmin, kmax
        self.window = window
        if window == "hanning":
            win = hanning_window(self.k_uniform, kmin, kmax, dk_win)
        elif window == "kaiser":
            win = kaiser_window(self.k_uniform, kmin, kmax, dk_win, beta)
        else:
            raise ValueError(f"unknown window {window!r}")
        win[self.k_uniform > self.k_model.max()] = 0.0
        win[self.k_uniform < self.k_model.min()] = 0.0
        self.weight = win * self.k_uniform ** kweight
        self.R = r_grid(nfft, dk)
        idx = np.searchsorted(self.k_model, self.k_uniform) - 1
        idx = np.clip(idx, 0, self.k_model.size - 2)
        span = np.maximum(self.k_model[idx + 1] - self.k_model[idx], 1e-12)
        frac = np.clip((self.k_uniform - self.k_model[idx]) / span, 0.0, 1.0)
        inside = (self.k_uniform >= self.k_model[0]) & (self.k_uniform <= self.k_model[-1])
        self._idx = idx
        self._frac = frac * inside
        self._inside = inside.astype(np.float64)
        self._w = self.weight
        self._norm = dk / np.sqrt(np.pi)
        self._basis = {}

    # ---------------------------------------------------------- set-up data
    def coefficients(self):
        """(n0, idx, frac, w) over the window's support: the uniform-grid
        indices n0 .. n0+len-1 where inside * weight is non-zero."""
        wt = self._w * self._inside
        nz = np.nonzero(wt)[0]
        if nz.size == 0:
            return 0, np.zeros(1, np.int32), np.zeros(1), np.zeros(1)
        n0, n1 = int(nz[0]), int(nz[-1]) + 1
        return (n0, self._idx[n0:n1].astype(np.int32), self._frac[n0:n1].copy(),
                wt[n0:n1].copy())

    def basis(self, bins=None):
        """Complex (nk, nbins): chi(R)[bins] = chi(k) @ basis."""
        key = None if bins is None else tuple(np.asarray(bins).tolist())
        if key in self._basis:
            return self._basis[key]
        bins = np.arange(self.nfft // 2) if bins is None else np.asarray(bins, np.int64)
        n0, idx, frac, w = self.coefficients()
        n = n0 + np.arange(idx.size)
        ph = (np.outer(n, bins) % self.nfft) * (2.0 * np.pi / self.nfft)
        F = (np.cos(ph) - 1j * np.sin(ph)) * self._norm            # (nwin, nbins)
        B = np.zeros((self.k_model.size, bins.size), complex)
        np.add.at(B, idx, ((1.0 - frac) * w)[:, None] * F)
        np.add.at(B, idx + 1, (frac * w)[:, None] * F)
        self._basis[key] = B
        return B

    def window_mask(self, rmin, rmax):
        return (self.R >= rmin) & (self.R <= rmax)

    def n_independent(self, rmin, rmax):
        return 2 * (self.kmax - self.kmin) * (rmax - rmin) / np.pi + 2

    # ---------------------------------------------------------- evaluation
    def to_R(self, chi, bins=None, precision=0):
        """chi (..., nk) -> complex chi(R) (..., nbins), default all nfft/2.
        The basis is uploaded to the device once per set of bins."""
        key = None if bins is None else tuple(np.asarray(bins).tolist())
        dev = self.__dict__.setdefault("_basis_dev", {})
        if key not in dev:
            dev[key] = basis_to_device(self.basis(bins))
        return apply_basis(chi, self.basis(bins), precision, Bd=dev[key])

    def magnitude(self, chi):
        out = self.to_R(chi)
        return np.abs(out) if isinstance(out, np.ndarray) else out.abs()

    def resample(self, chi):
        """chi (..., nk) -> (..., nfft) on the uniform grid (set-up check)."""
        x = np.asarray(chi)
        a = x[..., self._idx]
        b = x[..., self._idx + 1]
        return (a + (b - a) * self._frac) * self._inside


def basis_to_device(B):
    """The (nk, nb) complex basis as the (nk, 2 nb) FP64 device array the
    contraction takes (re, im interleaved)."""
    import torch
    nk = B.shape[0]
    return torch.from_numpy(np.ascontiguousarray(
        np.stack([B.real, B.imag], axis=-1).reshape(nk, -1))).to("cuda")


def apply_basis(chi, B, precision=0, Bd=None):
    """Device contraction of chi (..., nk) with a complex basis (nk, nb);
    Bd: its device copy from basis_to_device, when already uploaded."""
    import torch
    N.require_cuda()
    host = not (isinstance(chi, torch.Tensor) and chi.is_cuda)
    x = torch.as_tensor(np.asarray(chi) if host else chi).to("cuda", torch.float64).contiguous()
    lead = tuple(x.shape[:-1])
    nk = x.shape[-1]
    rows = int(np.prod(lead)) if lead else 1
    if Bd is None:
        Bd = basis_to_device(B)
    nb = B.shape[1]
    out = torch.empty((rows, 2 * nb), dtype=torch.float64, device="cuda")
    nsc = int(N.lib().chx_ft_batch_scratch_bytes(rows, nk, nb, precision))
    scr = torch.empty(max(nsc, 1), dtype=torch.uint8, device="cuda")
    N.call("chx_ft_batch", N.ptr(x), rows, nk, N.ptr(Bd), nb, precision, N.ptr(out), N.ptr(scr),
           nsc, N.stream())
    if precision in (2, 3) and int(scr[:4].view(torch.int32).item()):
        raise N.ChxError("chx_ft_batch: the tensor-core contraction gave up a bounded wait")
    z = torch.view_as_complex(out.view(rows, nb, 2)).reshape(lead + (nb,))
    return z.cpu().numpy() if host else z


class EdgeTransforms:
    """The k -> R channels of a multi-edge fit, ordered edge-major: for each
    absorber edge, one FourierTransform per k weight, all on one R grid.

    Evaluation is one device contraction per edge: that edge's chi(k) rows
    against the bases of all its channels laid side by side, (nk, nkw * nbins),
    so a whole spectrum set costs nsp launches instead of one per channel.
    An optional fixed chi_extra (nsp, nk) is added before transforming (the
    composition-averaged multiple-scattering term of the reference's fits).

    The samplers read the flat channel list `fts` and the channel -> edge map
    `chan_edge`; the reference's own adapter (chimera/multift.py) exposes the
    same two names, so either object can be handed to them."""

    def __init__(self, per_edge, chi_extra=None):
        per_edge = [list(ch) for ch in per_edge]
        if not per_edge or any(not ch for ch in per_edge):
            raise ValueError("every edge needs at least one channel")
        self.per_edge = per_edge
        self.fts = [f for ch in per_edge for f in ch]
        self.nsp = len(per_edge)
        self.nchan = len(self.fts)
        self.chan_edge = np.repeat(np.arange(self.nsp, dtype=np.int32),
                                   [len(ch) for ch in per_edge]).astype(np.int32)
        self.R = np.asarray(self.fts[0].R)
        if any(f.nfft != self.fts[0].nfft or f.dk != self.fts[0].dk for f in self.fts):
            raise ValueError("all channels must share one R grid (nfft, dk)")
        self.chi_extra = (None if chi_extra is None
                          else np.ascontiguousarray(chi_extra, np.float64))
        self._edge_dev = {}

    @classmethod
    def build(cls, k_axes, kmin, kmax, kweights, nsp=None, window="hanning", dk_win=1.0,
              beta=4.0, chi_extra=None):
        """Channels for every edge and k weight. k_axes: one model k axis for
        all edges, or a list with one per edge (edges fitted with their own
        E0 shift)."""
        if isinstance(k_axes, (list, tuple)):
            axes = [np.asarray(k, float) for k in k_axes]
        else:
            if nsp is None:
                raise ValueError("nsp is needed with a single k axis")
            axes = [np.asarray(k_axes, float)] * int(nsp)
        per_edge = [[FourierTransform(k, kmin, kmax, w, dk_win=dk_win, window=window, beta=beta)
                     for w in kweights] for k in axes]
        return cls(per_edge, chi_extra=chi_extra)

    def edge_basis(self, e, bins=None):
        """Complex (nk, nkw * nbins): the edge's channels side by side."""
        return np.concatenate([f.basis(bins) for f in self.per_edge[e]], axis=1)

    def to_R(self, chi, bins=None, precision=0):
        """chi (..., nsp, nk) -> complex chi(R) (..., nchan, nbins)."""
        import torch
        host = not (isinstance(chi, torch.Tensor) and chi.is_cuda)
        x = torch.as_tensor(np.asarray(chi) if host else chi).to("cuda", torch.float64)
        if self.chi_extra is not None:
            x = x + torch.as_tensor(self.chi_extra, device="cuda")
        key = None if bins is None else tuple(np.asarray(bins).tolist())
        nb = self.fts[0].nfft // 2 if bins is None else len(key)
        parts = []
        for e, ch in enumerate(self.per_edge):
            B = self.edge_basis(e, bins)
            if (e, key) not in self._edge_dev:
                self._edge_dev[(e, key)] = basis_to_device(B)
            z = apply_basis(x[..., e, :].contiguous(), B, precision, Bd=self._edge_dev[(e, key)])
            parts.append(z.reshape(z.shape[:-1] + (len(ch), nb)))
        out = torch.cat(parts, dim=-2)
        return out.cpu().numpy() if host else out

    def window_mask(self, rmin, rmax):
        return (self.R >= rmin) & (self.R <= rmax)

    def n_independent(self, rmin, rmax):
        kmin = min(f.kmin for f in self.fts)
        kmax = max(f.kmax for f in self.fts)
        return 2 * (kmax - kmin) * (rmax - rmin) / np.pi + 2


class WindowSums:
    """The fused form of the transform (chx_ft_window_sums) for a fixed basis
    B (nk, nbins), target (nbins, complex) and weights (nbins; 1 / sigma^2 on
    the fit window, 0 elsewhere): for each row of chi (rows, nk), with m its
    chi(R), the sums (rows, 7) = (Re<m,t>, <m,m>, sum w |s0 m - t|^2,
    sum w Re(m (s0 m - t)*), sum w |m|^2, sum |s0 m - t|^2,
    sum Re(m (s0 m - t)*)) over the window, chi(R) itself never written; precision 2 (split BF16) or 3 (TF32) on the tensor cores. The
    device copies of basis, target and weights and the scratch are made once,
    so `__call__` is one launch pair on the current stream."""

    def __init__(self, B, target, weight, rows, precision=2, s0=1.0, Bd=None):
        import torch
        N.require_cuda()
        self.nk, self.nb = B.shape
        self.rows, self.precision, self.s0 = int(rows), int(precision), float(s0)
        self.Bd = basis_to_device(B) if Bd is None else Bd
        t = np.asarray(target)
        self.td = torch.from_numpy(np.ascontiguousarray(
            np.stack([t.real, t.imag], -1).reshape(-1), np.float64)).to("cuda")
        self.wd = torch.from_numpy(np.ascontiguousarray(weight, np.float64)).to("cuda")
        self.nsc = int(N.lib().chx_ft_window_sums_scratch_bytes(self.rows, self.nk, self.nb,
                                                                self.precision))
        self.scr = torch.empty(max(self.nsc, 1), dtype=torch.uint8, device="cuda")
        self.out = torch.empty((self.rows, 7), dtype=torch.float64, device="cuda")

    def __call__(self, x):
        """x: (rows, nk) FP64 CUDA tensor -> (rows, 7) CUDA tensor (reused)."""
        N.call("chx_ft_window_sums", N.ptr(x), self.rows, self.nk, N.ptr(self.Bd), self.nb,
               N.ptr(self.td), N.ptr(self.wd), self.s0, self.precision, N.ptr(self.out),
               N.ptr(self.scr), self.nsc, N.stream())
        return self.out

    def device_error(self):
        """The scratch's error word (non-zero: a bounded wait ran out)."""
        import torch
        return int(self.scr[:4].view(torch.int32).item())

    @staticmethod
    def chi2(sums, s0=1.0, profile=True):
        """Per row: the profiled scale s (Re<m,t> / <m,m>, or 1),
        sum w |s m - t|^2 and sum |s m - t|^2 (the R-factor's numerator) from
        the anchored sums."""
        nu, dn, R, Q, P, Ru, Qu = (sums[..., q] for q in range(7))
        s = nu / dn if profile else 1.0 + 0.0 * nu
        ds = s - s0
        return s, R + 2.0 * ds * Q + ds * ds * P, Ru + 2.0 * ds * Qu + ds * ds * dn


def window_sums(chi, B, target, weight, precision=2, s0=1.0, Bd=None):
    """One-off chx_ft_window_sums (WindowSums) on chi (..., nk), host or
    device; returns (..., 7) of the same kind."""
    import torch
    host = not (isinstance(chi, torch.Tensor) and chi.is_cuda)
    x = torch.as_tensor(np.asarray(chi) if host else chi).to("cuda", torch.float64).contiguous()
    lead = tuple(x.shape[:-1])
    rows = int(np.prod(lead)) if lead else 1
    ws = WindowSums(B, target, weight, rows, precision, s0, Bd=Bd)
    out = ws(x.reshape(rows, -1)).clone()
    if ws.device_error():
        raise N.ChxError("chx_ft_window_sums: the tensor-core contraction gave up a bounded wait")
    out = out.reshape(lead + (7,))
    return out.cpu().numpy() if host else out
