"""Scattering tables: f(k), delta(k), lambda(k) on the model's k grid.

`ScatteringTables` has the reference's layout (exafs_gpu/scattering.py:48-105):
f (nsp, nk) by scatterer, delta (nsp, nsp, nk) by [absorber, scatterer],
lam (nk), k (nk), s02.

`smooth_tables` are the synthetic tables the benchmark configurations name:
|f_b(k)| = Z_b exp(-0.1 k) / k, delta_ab(k) = -0.8 k + 2, and the mean free
path lambda(k) = 59.57 / max(k, 1)^2 + 0.794 k clipped to [4, 30] A, the
"universal curve" stand-in of exafs_gpu/scattering.py:274-275. They are not
physical (f is 10-30x larger than a real backscattering amplitude), so the
absolute chi(k) tolerances measured on them are correspondingly strict.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

_SYMBOLS = ("H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn "
            "Ga Ge As Se Br Kr Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce "
            "Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi").split()
Z_TABLE = {s: i + 1 for i, s in enumerate(_SYMBOLS)}


@dataclass
class ScatteringTables:
    k: np.ndarray
    f: np.ndarray
    delta: np.ndarray
    lam: np.ndarray
    s02: float = 0.85
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        n = self.f.shape[0]
        assert self.f.shape == (n, self.k.size), "f must be (nsp, nk)"
        assert self.delta.shape == (n, n, self.k.size), "delta must be (nsp, nsp, nk)"
        assert self.lam.shape == self.k.shape

    @property
    def nsp(self):
        return self.f.shape[0]

    def as_float64(self):
        return (np.ascontiguousarray(self.k, np.float64), np.ascontiguousarray(self.f, np.float64),
                np.ascontiguousarray(self.delta, np.float64),
                np.ascontiguousarray(self.lam, np.float64))


def mean_free_path(k):
    kk = np.maximum(np.asarray(k, float), 1e-6)
    return np.clip(59.57 / np.maximum(kk, 1.0) ** 2 + 0.794 * kk, 4.0, 30.0)


def smooth_tables(k, elements, s02=0.85):
    """The benchmark's seeded smooth tables (see module docstring)."""
    k = np.asarray(k, np.float64)
    kk = np.maximum(k, 1e-6)
    els = tuple(elements)
    n = len(els)
    f = np.array([Z_TABLE[e] * np.exp(-0.1 * kk) / kk for e in els])
    delta = np.broadcast_to(-0.8 * kk + 2.0, (n, n, k.size)).copy()
    return ScatteringTables(k=k, f=f, delta=delta, lam=mean_free_path(k), s02=s02,
                            meta=dict(route="smooth", elements=els))


def uniform_k(kmin=2.0, kmax=14.0, dk=0.05):
    """The benchmark k grid: 2-14 A^-1 at 0.05 (241 points)."""
    n = int(round((kmax - kmin) / dk)) + 1
    return kmin + dk * np.arange(n)
