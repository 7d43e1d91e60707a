"""CPU restatement of the pair-count calibration objective (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this module,
as the checker of chimera_b200.shellmodel / chx_shell_rfactor; it is never
called by the library.

The reference's ShellModel.r_factor (chimera/shellmodel.py:427-440) for one
parameter set in the flat layout of chx_shell_rfactor:
  basis    B[a,b,s](k), shellmodel.py:290-336 (no physical per-pair tables)
  chi_k    shellmodel.py:411-413 (absorber counts :388-390)
  chi_ms   shellmodel.py:338-356 over multiscat.py:133-145 (chi_fast)
  to_R     exafs_gpu/fourier.py:21-83 on the k axis of model.py:120-130, the
           FFT written as a direct DFT on the requested bins
  fit      model.py:497-545 (fit_scales with one amplitude per edge, r_factor)
Pinned against the reference itself: tests/golden/shellmodel.npz, made by
tests/golden/make_shellmodel_golden.py from the reference's own ShellModel.
"""
from __future__ import annotations

import numpy as np


def unpack(x, nsp, nshell):
    x = np.asarray(x, float)
    nn = nsp * nsp
    o = 6
    p = dict(a0=x[0], sigma_scale=x[1], ms_amp=x[2], ms_c=x[3], kmin=x[4], kmax=x[5])
    p["dE0"] = x[o:o + nsp]; o += nsp
    p["sigma_shell_scale"] = x[o:o + nshell]; o += nshell
    p["dr"] = x[o:o + nn].reshape(nsp, nsp); o += nn
    p["c3"] = x[o:o + nshell]; o += nshell
    p["c4"] = x[o:o + nshell]; o += nshell
    p["sigma_pair"] = x[o:o + nn].reshape(nsp, nsp); o += nn
    p["ms_amp_edge"] = x[o:o + nsp]; o += nsp
    assert o == x.size
    return p


def basis(p, k, f, delta, lam, shells_ref, sigma2_ref, a0_ref, s02):
    """shellmodel.py:290-336, delta (nsp*nsp, nk)."""
    nsp, nshell = f.shape[0], len(shells_ref)
    r_s = np.asarray(shells_ref) * (p["a0"] / a0_ref)
    s2 = np.asarray(sigma2_ref) * p["sigma_scale"] * p["sigma_shell_scale"]
    B = np.zeros((nsp, nsp, nshell, k.size))
    k2, k3, k4 = k ** 2, k ** 3, k ** 4
    for s in range(nshell):
        amp4 = (2.0 / 3.0) * k4 * p["c4"][s]
        for a in range(nsp):
            for b in range(nsp):
                r = r_s[s] + (p["dr"][a, b] if s == 0 else 0.0)
                s2ab = s2[s] * (p["sigma_pair"][a, b] if s == 0 else 1.0)
                ph3 = (4.0 / 3.0) * k3 * p["c3"][s]
                B[a, b, s] = (s02 * f[b] / (k * r * r)
                              * np.exp(-2.0 * r / lam - 2.0 * k2 * s2ab + amp4)
                              * np.sin(2.0 * k * r + delta[a * nsp + b] - ph3))
    return B


def chi_ms(p, k, ms, shells_ref, sigma2_ref, a0_ref, s02, nsp):
    """shellmodel.py:338-356 + multiscat.py:133-145. ms: dict of absorber,
    reff, deg (npath), F, D, L (npath, nk), dnn; None for no MS."""
    if ms is None:
        return 0.0
    r_nn = shells_ref[0] * (p["a0"] / a0_ref)
    s2nn = sigma2_ref[0] * p["sigma_scale"] * p["sigma_shell_scale"][0]
    a_scale = r_nn / ms["dnn"]
    out = np.zeros((nsp, k.size))
    for e in range(nsp):
        sel = ms["absorber"] == e
        r = (ms["reff"][sel] * a_scale)[:, None]
        s2 = p["ms_c"] * s2nn * r / (2.0 * r_nn)
        term = (ms["deg"][sel][:, None] * s02 * ms["F"][sel] / np.maximum(k[None, :] * r ** 2, 1e-12)
                * np.exp(-2.0 * r / np.maximum(ms["L"][sel], 1e-6) - 2.0 * k[None, :] ** 2 * s2)
                * np.sin(2.0 * k[None, :] * r + ms["D"][sel]))
        out[e] = p["ms_amp"] * term.sum(axis=0)
    return out * np.asarray(p["ms_amp_edge"])[:, None]


def hanning(k, kmin, kmax, dk_win):
    w = np.zeros_like(k)
    w[(k >= kmin + dk_win / 2) & (k <= kmax - dk_win / 2)] = 1.0
    lo = (k > kmin - dk_win / 2) & (k < kmin + dk_win / 2)
    w[lo] = 0.5 * (1 + np.sin(np.pi * (k[lo] - kmin) / dk_win))
    hi = (k > kmax - dk_win / 2) & (k < kmax + dk_win / 2)
    w[hi] = 0.5 * (1 - np.sin(np.pi * (k[hi] - kmax) / dk_win))
    return w


def to_R(chi_e, k_model, kmin, kmax, w, dk_win, bins, nfft=2048, dk=0.05):
    """exafs_gpu/fourier.py:21-83 on bins of the FFT grid (direct DFT)."""
    ku = np.arange(nfft) * dk
    win = hanning(ku, kmin, kmax, dk_win)
    win[ku > k_model.max()] = 0.0
    win[ku < k_model.min()] = 0.0
    weight = win * ku ** w
    idx = np.clip(np.searchsorted(k_model, ku) - 1, 0, k_model.size - 2)
    span = np.maximum(k_model[idx + 1] - k_model[idx], 1e-12)
    inside = (ku >= k_model[0]) & (ku <= k_model[-1])
    frac = np.clip((ku - k_model[idx]) / span, 0.0, 1.0) * inside
    a, b = chi_e[idx], chi_e[idx + 1]
    x = (a + (b - a) * frac) * inside * weight
    n = np.arange(nfft)
    ph = 2.0 * np.pi * ((np.outer(bins, n)) % nfft) / nfft
    return (x[None, :] * (np.cos(ph) - 1j * np.sin(ph))).sum(1) * dk / np.sqrt(np.pi)


def r_factor(x, N, model, data, bins, kweight, magnitude=False, ms=None):
    """(R-factor, per-edge amplitudes) of one flat parameter row. `model`:
    dict k, f, delta, lam, shells_ref, shell_mult, sigma2_ref, a0_ref, s02,
    dk_win, etok; data (nchan, nbin) on the fitted bins."""
    k = model["k"]
    nsp, nshell = model["f"].shape[0], len(model["shells_ref"])
    p = unpack(x, nsp, nshell)
    B = basis(p, k, model["f"], model["delta"], model["lam"], model["shells_ref"],
              model["sigma2_ref"], model["a0_ref"], model["s02"])
    cnt = np.maximum(np.asarray(N).sum(axis=(1, 2)) / np.sum(model["shell_mult"]), 1e-30)
    chi = np.einsum("abs,absk->ak", N, B) / cnt[:, None] + chi_ms(
        p, k, ms, model["shells_ref"], model["sigma2_ref"], model["a0_ref"], model["s02"], nsp)
    m = []
    for e in range(nsp):
        km = np.sqrt(np.maximum(k ** 2 - model["etok"] * p["dE0"][e], 1e-4))
        for w in kweight:
            m.append(to_R(chi[e], km, p["kmin"], p["kmax"], w, model["dk_win"], bins))
    m = np.array(m)
    if magnitude:
        m = np.abs(m)
    d = np.asarray(data)
    edge = np.repeat(np.arange(nsp), len(kweight))
    num = np.real((np.conj(m) * d).sum(axis=1))
    den = np.real((np.conj(m) * m).sum(axis=1))
    num = np.bincount(edge, num, nsp)[edge]
    den = np.bincount(edge, den, nsp)[edge]
    sc = num / np.maximum(den, 1e-30)
    rf = (np.abs(m * sc[:, None] - d) ** 2).sum() / max((np.abs(d) ** 2).sum(), 1e-30)
    return float(rf), sc[[int(np.argmax(edge == e)) for e in range(nsp)]]
