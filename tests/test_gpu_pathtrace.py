"""chx_path_trace (curved-wave path trace) against the reference's own
trace_numpy (tests/golden/pathtrace.npz) and the CPU evaluation."""
import numpy as np
import pytest

from conftest import golden
from oracle import pathtrace as OP

pytestmark = pytest.mark.gpu


def test_traces_match_reference(cuda):
    """Five paths (single scattering, triangle, general four-leg, collinear
    forward, back-and-forth) at 8 energies each, lmax 10-14 per energy: one
    launch; every trace equals the reference's trace_numpy to 1e-9 relative."""
    from chimera_b200.pathtrace import path_trace
    g = golden("pathtrace.npz")
    t = 0.5 * (g["S"] - 1.0)
    ie = g["energies"]
    sites = [g["sites"][q, :n] for q, n in enumerate(g["nsc"])]
    types = [tuple(g["types"][q, :n]) for q, n in enumerate(g["nsc"])]
    tr = path_trace(sites, types, g["p"][ie], t[:, ie], g["lmax"])
    rel = np.abs(tr - g["trace"]) / np.abs(g["trace"])
    assert rel.max() <= 1e-9, rel.max()


def test_high_lmax_matches_cpu_evaluation(cuda):
    """A general five-leg path at lmax 24 and 30 (beyond the fixtures): the
    kernel equals the CPU evaluation with dense Wigner matrices to 1e-9."""
    from chimera_b200.pathtrace import path_trace
    g = golden("pathtrace.npz")
    rng = np.random.default_rng(5)
    nl = 32
    kb = 6.0
    S = np.exp(2j * (0.8 * np.exp(-(np.arange(nl) / 14.0) ** 2)[None, :]
                     * np.array([[1.0], [1.2]]) + 0.01j))
    t = 0.5 * (S - 1.0)[:, None, :]
    p = np.array([kb + 0.03j])
    site = rng.normal(0, 4.0, (4, 3)) + np.array([4.0, 0, 0])
    for lmax in (24, 30):
        got = path_trace([site], [(0, 1, 1, 0)], p, t, np.array([[lmax]]))[0, 0]
        ref = OP.trace(site, (0, 1, 1, 0), p[0], t[:, 0], lmax)
        assert abs(got - ref) <= 1e-9 * abs(ref), (lmax, got, ref)


def test_bad_type_is_nan_and_isolated(cuda):
    from chimera_b200.pathtrace import path_trace
    g = golden("pathtrace.npz")
    t = 0.5 * (g["S"] - 1.0)
    ie = g["energies"][:2]
    sites = [g["sites"][0, :1], g["sites"][0, :1]]
    tr = path_trace(sites, [(0,), (7,)], g["p"][ie], t[:, ie], g["lmax"][:2, :2])
    assert np.isnan(tr[1]).all()
    assert np.allclose(tr[0], g["trace"][0, :2], rtol=1e-9, atol=0)
