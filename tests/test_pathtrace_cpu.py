"""The path-trace tables and geometry (chimera_b200.pathtrace) and the CPU
evaluation (oracle) against the reference's own trace_numpy."""
import math

import numpy as np
import pytest

from conftest import golden
from chimera_b200 import pathtrace as PT
from oracle import pathtrace as OP


def test_small_d_identities():
    """d^l(beta) is orthogonal, d^l(0) = 1, and the Delta factorisation
    d_{mm'}(beta) = i^(m-m') sum_m'' Delta_{m''m} Delta_{m''m'} e^{-i m'' beta}
    holds for l up to 12."""
    for l in (0, 1, 2, 5, 12):
        d = PT.small_d(l, 0.7)
        assert np.allclose(d @ d.T, np.eye(2 * l + 1), atol=1e-12)
        assert np.allclose(PT.small_d(l, 0.0), np.eye(2 * l + 1), atol=1e-13)
        D = PT.small_d(l, math.pi / 2)
        m = np.arange(-l, l + 1)
        rec = ((1j ** ((m[:, None] - m[None, :]) % 4))
               * np.einsum("km,kn,k->mn", D, D, np.exp(-1j * m * 0.7)))
        assert np.allclose(rec.real, d, atol=1e-12) and np.abs(rec.imag).max() < 1e-12


def test_gaunt_runs_selection_rules():
    off, cnt, lpp, A = PT.propagator_runs(6)
    # l'' runs only over |l - l'| .. l + l' with l + l' + l'' even
    for (m, lp, l) in [(0, 0, 0), (1, 2, 3), (2, 4, 4), (0, 6, 5)]:
        o, c = off[m, lp, l], cnt[m, lp, l]
        assert np.all((lpp[o:o + c] + l + lp) % 2 == 0)
        assert np.all((lpp[o:o + c] >= abs(l - lp)) & (lpp[o:o + c] <= l + lp))
    # (l', l) = (0, 0): A = 4 pi C(00,00,00) sqrt(1/4pi) = 1
    assert np.isclose(A[off[0, 0, 0]], 1.0)


def test_oracle_trace_matches_reference():
    """Single scattering, triangle, general four-leg, collinear forward and
    back-and-forth paths at lmax 10-14: the CPU trace equals the reference's
    trace_numpy to 1e-9 relative."""
    g = golden("pathtrace.npz")
    t = 0.5 * (g["S"] - 1.0)
    for q in range(len(g["nsc"])):
        n = int(g["nsc"][q])
        for j, ie in enumerate(g["energies"][::2]):
            jj = 2 * j
            got = OP.trace(g["sites"][q, :n], g["types"][q, :n], g["p"][ie], t[:, ie],
                           int(g["lmax"][q, jj]))
            ref = g["trace"][q, jj]
            assert abs(got - ref) <= 1e-9 * abs(ref), (q, ie, got, ref)
