"""Golden vectors of the curved-wave path trace, from the reference.

    python tests/golden/make_pathtrace_golden.py /path/to/reference   (or CHIMERA_REFERENCE=...)

Builds a `PhaseShifts` (exafs_gpu/abinitio/phaseshift.py:54-67) of two
scatterer types with smooth synthetic complex phase shifts on 24 energies
(k 2-14 A^-1, momenta with a small imaginary part), and evaluates the
reference's own `pathsum.trace_numpy` (exafs_gpu/abinitio/pathsum.py:106-126)
for five paths: single scattering, a triangle, a general four-leg path, a
collinear forward-scattering path and a back-and-forth four-leg path (the two
Euler-angle special cases), at each path's lmax_per_energy (capped at 14).
Saves the phase shifts, the paths and the traces (pathtrace.npz).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_path  # noqa: E402

REF = reference_path()
sys.path.insert(0, os.path.join(HERE, "_stub"))
sys.path.insert(0, REF)

from exafs_gpu.abinitio import pathsum as PS        # noqa: E402
from exafs_gpu.abinitio.phaseshift import PhaseShifts  # noqa: E402

BOHR = 0.529177210903


def phase_shifts(nE=24, nl=26, seed=0):
    k = np.linspace(2.0, 14.0, nE)
    kb = k * BOHR
    p = kb + 1j * (0.02 + 0.002 * kb)
    rng = np.random.default_rng(seed)
    S = np.empty((2, nE, nl), complex)
    l = np.arange(nl)
    for t in range(2):
        r_mt = 2.3 + 0.3 * t
        amp = 0.9 + 0.25 * t
        for ie in range(nE):
            width = 0.75 * kb[ie] * r_mt + 1.0
            d = amp * np.exp(-(l / width) ** 2) * (1.0 + 0.05 * rng.standard_normal())
            d = d + 1j * 0.02 * np.exp(-(l / width) ** 2)
            S[t, ie] = np.exp(2j * d)
    return PhaseShifts(k=k, energy=k ** 2 / 3.80998 / 27.211386, p=p, S=S,
                       labels=["A", "B"], gamma_ch=0.0, r_mt=np.array([2.3, 2.6]))


def main():
    ph = phase_shifts()
    a = 2.54 / BOHR                                    # nearest-neighbour distance, bohr
    v = np.array([[a, 0, 0], [0, a, 0], [0, 0, a]]) / np.sqrt(2.0)
    paths = [
        PS.Path(np.array([[0.3, 0.4, 1.0]]) * a / np.linalg.norm([0.3, 0.4, 1.0]), (0,), 12.0),
        PS.Path(np.array([v[0] + v[1], v[1] + v[2]]), (0, 1), 24.0),
        PS.Path(np.array([[a, 0.2 * a, 0.1 * a], [0.9 * a, 1.1 * a, -0.3 * a],
                          [0.1 * a, 0.8 * a, 0.5 * a]]), (1, 0, 1), 48.0),
        PS.Path(np.array([[0, 0, a], [0, 0, 2 * a]]), (0, 1), 6.0),
        PS.Path(np.array([[a, 0, 0], [0, 0, 0.0 + 1e-9], [a, 0, 0]]) if False else
                np.array([[a, 0, 0], [2 * a, 0, 0], [a, 0, 0]]), (1, 0, 1), 6.0),
    ]
    energies = np.arange(0, ph.k.size, 3)
    maxs = max(len(pth.types) for pth in paths)
    sites = np.zeros((len(paths), maxs, 3))
    types = np.full((len(paths), maxs), -1, np.int32)
    nsc = np.array([len(pth.types) for pth in paths], np.int32)
    lmax = np.zeros((len(paths), energies.size), np.int32)
    tr = np.zeros((len(paths), energies.size), complex)
    for q, pth in enumerate(paths):
        sites[q, :nsc[q]] = pth.sites
        types[q, :nsc[q]] = pth.types
        lm = PS.lmax_per_energy(ph, pth.types, cap=14)
        for j, ie in enumerate(energies):
            lmax[q, j] = int(lm[ie])
            tr[q, j] = PS.trace_numpy(pth, ph, int(ie), int(lm[ie]))
    np.savez_compressed(os.path.join(HERE, "pathtrace.npz"), k=ph.k, p=ph.p, S=ph.S,
                        sites=sites, types=types, nsc=nsc, energies=energies, lmax=lmax,
                        trace=tr, degeneracy=np.array([pth.degeneracy for pth in paths]))
    print("wrote pathtrace.npz; lmax range", lmax.min(), lmax.max())
    print("traces", np.round(tr[:, ::3], 6))


if __name__ == "__main__":
    main()
