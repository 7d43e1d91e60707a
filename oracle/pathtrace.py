"""CPU evaluation of the curved-wave path trace (test infrastructure).

Only tests/ use this module, as the checker of chx_path_trace. It evaluates
Tr_{l=1} of the path product of exafs_gpu/abinitio/pathsum.py:106-126 with
dense matrices: the propagator g^m_{l'l}(p |a|) from the A runs of
chimera_b200.pathtrace and spherical Hankel functions by upward recurrence,
and every frame change as the full Wigner matrix e^{-i m alpha} d^l(beta)
e^{-i m' gamma} with d^l(beta) = exp(-i beta J_y) (no Delta factorisation, so
the kernel's two-product rotation is checked against an independent form).
Pinned against the reference's own trace_numpy: tests/golden/pathtrace.npz
(tests/golden/make_pathtrace_golden.py).
"""
from __future__ import annotations

import numpy as np

from chimera_b200 import pathtrace as PT


def hankel(lmax, x):
    """h_l(x) = j_l + i n_l, l = 0..lmax, complex x (upward recurrence)."""
    h = np.empty(lmax + 1, complex)
    e = np.exp(1j * x)
    h[0] = -1j * e / x
    if lmax >= 1:
        h[1] = -e / x * (1.0 + 1j / x)
    for l in range(1, lmax):
        h[l + 1] = (2 * l + 1) / x * h[l] - h[l - 1]
    return h


def propagate(v, lmax, x):
    off, cnt, lpp, A = PT.propagator_runs(lmax)
    h = hankel(2 * lmax, x)
    out = np.zeros_like(v)
    for m in range(-lmax, lmax + 1):
        am = abs(m)
        ls = np.arange(am, lmax + 1)
        g = np.zeros((ls.size, ls.size), complex)
        for i, lp in enumerate(ls):
            for j, l in enumerate(ls):
                o, c = off[am, lp, l], cnt[am, lp, l]
                g[i, j] = (A[o:o + c] * h[lpp[o:o + c]]).sum()
        idx = ls * ls + ls + m
        out[idx] = g @ v[idx]
    return out


def rotate(v, lmax, eul):
    a, b, c = eul
    out = np.empty_like(v)
    for l in range(lmax + 1):
        m = np.arange(-l, l + 1)
        D = np.exp(-1j * m * a)[:, None] * PT.small_d(l, b) * np.exp(-1j * m * c)[None, :]
        sl = slice(l * l, (l + 1) ** 2)
        out[sl] = D @ v[sl]
    return out


def trace(sites, types, p, t, lmax):
    """Tr_{l=1} of one path at one energy: p complex momentum, t (ntype, nl)."""
    lens, eul = PT.path_frames(sites)
    n = (lmax + 1) ** 2
    v = np.zeros((n, 3), complex)
    for c, mu in enumerate((-1, 0, 1)):
        v[2 + mu, c] = 1.0
    v = propagate(v, lmax, p * lens[0])
    for j, ty in enumerate(types):
        v = np.repeat(t[ty, :lmax + 1], 2 * np.arange(lmax + 1) + 1)[:, None] * v
        v = rotate(v, lmax, eul[j])
        v = propagate(v, lmax, p * lens[j + 1])
    v = rotate(v, lmax, eul[-1])
    return sum(v[2 + mu, c] for c, mu in enumerate((-1, 0, 1)))
