"""Curved-wave multiple-scattering path trace (exafs_gpu/abinitio/pathsum.py).

For a K edge, orientation averaged, a path absorber -> R_1 -> ... -> R_N ->
absorber contributes chi = Re[e^{2 i delta_c} Tr_{l=1} P] / 3 with the path
product P = G(a_N) t_N ... t_1 G(a_0) (pathsum.py:1-22): G the free
spherical-wave propagator along a leg, t_l = (e^{2 i delta_l} - 1)/2 the
scatterer's amplitudes. Every factor is applied in the leg's own frame, where
the propagator is diagonal in m,

    g^m_{l'l}(x) = sum_l'' A^m_{l'l l''} h_l''(x),
    A^m_{l'l l''} = 4 pi i^(l'+l''-l) C(lm, l'm, l''0) sqrt((2 l''+1)/(4 pi)),

with C the Gaunt integral of complex Condon-Shortley harmonics and h_l the
outgoing spherical Hankel function, and the change of frame between legs is a
Wigner rotation D(alpha, beta, gamma) = e^{-i m alpha} d^l(beta) e^{-i m'
gamma}, applied as two products with Delta^l = d^l(pi/2):
d^l_{mm'}(beta) = i^(m-m') sum_m'' Delta_{m''m} Delta_{m''m'} e^{-i m'' beta}
(the conventions of sphere.py:1-23).

Host side here: the A runs (Gauss-Legendre quadrature of normalised
associated Legendre functions, exact for these polynomial degrees), the
Delta^l matrices (the matrix exponential of J_y), the leg frames and the
zyz Euler angles of their changes. The trace itself is `chx_path_trace`:
one CTA per (energy, path), FP64 complex, state and Hankel functions in
shared memory.
"""
from __future__ import annotations

import ctypes as C
import math
from functools import lru_cache

import numpy as np

from . import _native as N

MAX_L = 40          # chx_path_trace's angular momentum cap


def legendre_normalised(lmax, x):
    """Theta_lm(x) = sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!) P_l^m(x) with the
    Condon-Shortley phase, [l, m, point] for 0 <= m <= l <= lmax (Y_lm =
    Theta_lm e^{i m phi}), by the standard normalised recursions in m then l."""
    x = np.atleast_1d(np.asarray(x, float))
    s = np.sqrt(np.clip(1.0 - x * x, 0.0, None))
    T = np.zeros((lmax + 1, lmax + 1, x.size))
    T[0, 0] = 0.5 / math.sqrt(math.pi)
    for m in range(1, lmax + 1):                     # diagonal
        T[m, m] = -math.sqrt((2.0 * m + 1.0) / (2.0 * m)) * s * T[m - 1, m - 1]
    for m in range(lmax):                            # first off-diagonal
        T[m + 1, m] = math.sqrt(2.0 * m + 3.0) * x * T[m, m]
    for m in range(lmax + 1):                        # upward in l
        for l in range(m + 2, lmax + 1):
            c1 = math.sqrt((4.0 * l * l - 1.0) / (l * l - m * m))
            c2 = math.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1.0) ** 2 - 1.0))
            T[l, m] = c1 * (x * T[l - 1, m] - c2 * T[l - 2, m])
    return T


@lru_cache(maxsize=4)
def propagator_runs(lmax):
    """A^m_{l'l l''} packed for the kernel: for every (|m|, l', l) with
    |m| <= l, l' <= lmax a run of (l'', A) over l'' = |l-l'| .. l+l' (step 2)
    with C != 0. Returns off, cnt ((lmax+1)^3 int32, [m][l'][l]), lpp (int32)
    and A (complex128)."""
    nq = 2 * lmax + 2                                # exact for degree <= 4 lmax + 3
    xg, wg = np.polynomial.legendre.leggauss(nq)
    T = legendre_normalised(2 * lmax, xg)
    n = lmax + 1
    off = np.zeros((n, n, n), np.int32)
    cnt = np.zeros((n, n, n), np.int32)
    L, A = [], []
    for m in range(n):
        for lp in range(m, n):
            for l in range(m, n):
                lpp = np.arange(abs(l - lp), l + lp + 1, 2)
                # C(lm, l'm, l''0) = 2 pi int Theta_lm Theta_l'm Theta_l''0 dx
                c = 2.0 * math.pi * (T[lpp, 0] * (T[l, m] * T[lp, m] * wg)[None, :]).sum(1)
                keep = np.abs(c) > 1e-15
                off[m, lp, l] = len(L)
                cnt[m, lp, l] = int(keep.sum())
                ph = np.array([1, 1j, -1, -1j])[(lp + lpp[keep] - l) % 4]
                A.extend((4.0 * math.pi * ph * c[keep]
                          * np.sqrt((2 * lpp[keep] + 1) / (4.0 * math.pi))).tolist())
                L.extend(lpp[keep].tolist())
    return off, cnt, np.array(L, np.int32), np.array(A, complex)


def jy(l):
    """J_y in the |l m> basis, m = -l..l."""
    m = np.arange(-l, l)
    up = np.sqrt(l * (l + 1.0) - m * (m + 1.0))      # <m+1|J+|m>
    Jp = np.diag(up, -1)
    return (Jp - Jp.T) / 2j


def small_d(l, beta):
    """d^l(beta) = exp(-i beta J_y), real."""
    from scipy.linalg import expm
    return expm(-1j * beta * jy(l)).real


@lru_cache(maxsize=4)
def delta_runs(lmax):
    """Delta^l = d^l(pi/2), l = 0..lmax: offsets (lmax+2,) int64 and a flat
    array with Delta^l[m''+l, m+l] at off[l] + (m''+l)(2l+1) + (m+l)."""
    off = np.zeros(lmax + 2, np.int64)
    parts = []
    for l in range(lmax + 1):
        parts.append(small_d(l, math.pi / 2).ravel())
        off[l + 1] = off[l] + (2 * l + 1) ** 2
    return off, np.concatenate(parts)


def frame_of(v):
    """R = Rz(phi) Ry(theta): the rotation taking z to v/|v|."""
    v = np.asarray(v, float)
    th = math.acos(max(-1.0, min(1.0, v[2] / np.linalg.norm(v))))
    phi = math.atan2(v[1], v[0])
    cz, sz, cy, sy = math.cos(phi), math.sin(phi), math.cos(th), math.sin(th)
    return (np.array([[cz, -sz, 0.0], [sz, cz, 0.0], [0.0, 0.0, 1.0]])
            @ np.array([[cy, 0.0, sy], [0.0, 1.0, 0.0], [-sy, 0.0, cy]]))


def euler_zyz(Q):
    """(alpha, beta, gamma) with Q = Rz(alpha) Ry(beta) Rz(gamma); at
    beta = 0 or pi only alpha +- gamma is defined and gamma is set to 0."""
    Q = np.asarray(Q, float)
    beta = math.acos(max(-1.0, min(1.0, Q[2, 2])))
    if abs(math.sin(beta)) > 1e-10:
        return math.atan2(Q[1, 2], Q[0, 2]), beta, math.atan2(Q[2, 1], -Q[2, 0])
    if Q[2, 2] > 0:
        return math.atan2(Q[1, 0], Q[0, 0]), beta, 0.0
    return math.atan2(-Q[1, 0], -Q[0, 0]), beta, 0.0


def path_frames(sites):
    """Leg lengths (N+1,) and the Euler angles (N+1, 3) of the frame changes
    Q_j = R_j^T R_{j-1} (j = 1..N) and the closing R_0^T R_N, for scatterers
    `sites` (N, 3) with the absorber at the origin."""
    pts = np.vstack([np.zeros(3), np.asarray(sites, float), np.zeros(3)])
    legs = np.diff(pts, axis=0)
    R = [frame_of(a) for a in legs]
    eul = [euler_zyz(R[j].T @ R[j - 1]) for j in range(1, len(R))]
    eul.append(euler_zyz(R[0].T @ R[-1]))
    return np.linalg.norm(legs, axis=1), np.array(eul)


BUCKETS = (8, 16, 24, 32, MAX_L)     # table sizes energies are grouped by
_DEV_TABLES = {}


def _tables_on_device(cap):
    """Device copies of the propagator runs and Delta blocks for lmax <= cap."""
    if cap not in _DEV_TABLES:
        off, cnt, lpp, A = propagator_runs(cap)
        doff, dflat = delta_runs(cap)
        _DEV_TABLES[cap] = dict(
            goff=N.to_dev(off), gcnt=N.to_dev(cnt), glpp=N.to_dev(lpp),
            gA=N.to_dev(np.ascontiguousarray(np.stack([A.real, A.imag], -1))),
            doff=N.to_dev(doff), dflat=N.to_dev(dflat))
    return _DEV_TABLES[cap]


def path_trace(sites_list, types_list, p, t, lmax, stream=None):
    """Tr_{l=1} of every path's product at every energy, complex (npath, nE),
    on the device. sites_list: per path (N, 3) scatterer positions (bohr);
    types_list: per path N type indices into t; p (nE,) complex momenta
    (bohr^-1); t (ntype, nE, nl) complex amplitudes; lmax (npath, nE).
    Energies are grouped by their largest lmax into table sizes of BUCKETS,
    one launch each, so that low-lmax energies run with small shared-memory
    footprints (more CTAs per SM)."""
    import torch
    lmax = np.asarray(lmax, np.int32)
    npath, ne = lmax.shape
    Lc = int(lmax.max())
    t = np.asarray(t, complex)
    if Lc > MAX_L or Lc + 1 > t.shape[2] or int(lmax.min()) < 1:
        raise ValueError(f"lmax {Lc} outside 1..{MAX_L} or beyond the phase shifts")
    maxs = max(len(ty) for ty in types_list)
    nsc = np.array([len(ty) for ty in types_list], np.int32)
    typ = np.zeros((npath, maxs), np.int32)
    leg = np.zeros((npath, maxs + 1))
    eul = np.zeros((npath, maxs + 1, 3))
    for q, (st, ty) in enumerate(zip(sites_list, types_list)):
        ls, eu = path_frames(st)
        typ[q, :len(ty)] = ty
        leg[q, :len(ls)] = ls
        eul[q, :len(eu)] = eu
    paths = dict(nsc=N.to_dev(nsc), typ=N.to_dev(typ), leg=N.to_dev(leg), eul=N.to_dev(eul))
    p = np.asarray(p, complex)
    emax = lmax.max(axis=0)
    # table size per energy: the bucket of its largest lmax, no larger than
    # the phase shifts cover (lmax + 1 <= nl is checked above)
    cap_of = np.array([min(next(b for b in BUCKETS if b >= e), t.shape[2] - 1) for e in emax])
    result = np.empty((npath, ne), complex)
    outs = []
    for cap in sorted(set(cap_of.tolist())):
        sel = np.nonzero(cap_of == cap)[0]
        tab = _tables_on_device(cap)
        ts = t[:, sel]
        dev = dict(p=N.to_dev(np.stack([p[sel].real, p[sel].imag], -1).astype(np.float64)),
                   t=N.to_dev(np.ascontiguousarray(np.stack([ts.real, ts.imag], -1))),
                   lmax=N.to_dev(np.ascontiguousarray(lmax[:, sel])))
        out = torch.empty((npath, sel.size, 2), dtype=torch.float64, device="cuda")
        P = N.PathSet()
        P.npath, P.maxs, P.ne, P.ntype, P.nlt, P.glmax = (npath, maxs, int(sel.size),
                                                          t.shape[0], t.shape[2], cap)
        for k, v in list(paths.items()) + list(tab.items()) + list(dev.items()):
            setattr(P, k, N.dptr(v))
        N.call("chx_path_trace", C.byref(P), N.ptr(out),
               N.stream() if stream is None else stream)
        outs.append((sel, out, dev))
    for sel, out, _ in outs:
        o = out.cpu().numpy()
        result[:, sel] = o[..., 0] + 1j * o[..., 1]
    return result
