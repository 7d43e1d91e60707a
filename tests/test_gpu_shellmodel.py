"""chx_shell_rfactor (the pair-count calibration objective for a population)
against the reference's ShellModel.r_factor and the CPU restatement."""
import numpy as np
import pytest

from conftest import golden
from oracle import shellmodel as OS

pytestmark = pytest.mark.gpu


def device_model(g, ms=None):
    from chimera_b200.shellmodel import ShellModel
    sm = ShellModel(g["k"], (None, g["f"], g["delta"], g["lam"]), g["shells_ref"],
                    g["shell_mult"], g["sigma2_shell_ref"], int(g["natoms"]), float(g["a0_ref"]),
                    s02=float(g["s02"]), dk_win=float(g["dk_win"]), composition=(0.5, 0.5),
                    ms_paths=ms)
    sm.set_params(kweight=tuple(int(x) for x in g["kweight"]))
    return sm


def oracle_model(g):
    return dict(k=g["k"], f=g["f"], delta=g["delta"], lam=g["lam"], shells_ref=g["shells_ref"],
                shell_mult=g["shell_mult"], sigma2_ref=g["sigma2_shell_ref"],
                a0_ref=float(g["a0_ref"]), s02=float(g["s02"]), dk_win=float(g["dk_win"]),
                etok=float(g["etok"]))


@pytest.mark.parametrize("kind", ["complex", "magnitude"])
def test_population_matches_reference_r_factor(cuda, kind):
    """All 24 reference parameter sets in one launch: R-factors and per-edge
    amplitudes equal the reference's ShellModel.r_factor to 1e-9 relative
    (a direct DFT on the fitted bins in place of the FFT)."""
    g = golden("shellmodel.npz")
    sm = device_model(g)
    mag = kind == "magnitude"
    data = g["data_m"] if mag else g["data_c"]
    rf, sc = sm.r_factor_batch(g["N1"], data, g["mask"], g["idx"], g["params"])
    ref = g["rf_m"] if mag else g["rf_c"]
    rsc = g["scales_m"] if mag else g["scales_c"]
    assert np.allclose(rf, ref, rtol=1e-9, atol=0), np.abs(rf / ref - 1).max()
    assert np.allclose(sc, rsc, rtol=1e-9, atol=0)
    rf0, _ = sm.r_factor_batch(g["N0"], g["data_c"], g["mask"], g["idx"], g["params"])
    assert np.allclose(rf0, g["rf_n0"], rtol=1e-9, atol=0)
    # one member at a time gives the same, bit for bit (no cross-member state)
    one = [sm.r_factor_batch(g["N1"], data, g["mask"], g["idx"], x[None])[0][0]
           for x in g["params"][:4]]
    assert np.array_equal(np.array(one), rf[:4])


def synthetic_ms(g, seed=3):
    """A seeded averaged-MS path set on the model grid: 12 paths per
    absorber with smooth amplitudes, phases and mean free paths."""
    rng = np.random.default_rng(seed)
    k = g["k"]
    nsp = g["f"].shape[0]
    n = 12
    ab = np.repeat(np.arange(nsp), n)
    reff = rng.uniform(3.6, 5.4, nsp * n)
    deg = rng.integers(6, 48, nsp * n).astype(float)
    F = 0.1 * np.abs(g["f"][ab]) * rng.uniform(0.5, 1.5, (nsp * n, 1))
    D = -0.8 * k[None, :] + rng.uniform(0, 3, (nsp * n, 1))
    L = np.tile(g["lam"], (nsp * n, 1)) * rng.uniform(0.8, 1.2, (nsp * n, 1))
    return dict(absorber=ab, reff=reff, deg=deg, F=F, D=D, L=L,
                dnn=float(g["shells_ref"][0]))


def test_averaged_ms_term_matches_oracle(cuda):
    """With an averaged multiple-scattering path set (the reference's
    MSPaths.chi_fast form, scaled to the member's nearest-neighbour distance
    with its MS amplitude, c and per-edge amplitudes) the population's
    R-factors equal the CPU restatement to 1e-9 relative."""
    g = golden("shellmodel.npz")
    ms = synthetic_ms(g)
    sm = device_model(g, ms)
    X = g["params"].copy()
    rng = np.random.default_rng(9)
    X[:, 2] = np.exp(rng.uniform(np.log(0.3), np.log(2.5), len(X)))     # ms_amp
    X[:, 3] = np.exp(rng.uniform(np.log(0.4), np.log(3.0), len(X)))     # ms_c
    X[:, -2:] = np.exp(rng.uniform(-0.5, 0.5, (len(X), 2)))            # ms_amp_edge
    mask = g["mask"]
    rf, sc = sm.r_factor_batch(g["N1"], g["data_c"], mask, g["idx"], X)
    m = oracle_model(g)
    for q in range(0, len(X), 3):
        r, s = OS.r_factor(X[q], g["N1"], m, g["data_c"][:, mask], g["idx"][mask],
                           g["kweight"], ms=ms)
        assert abs(rf[q] - r) <= 1e-9 * r, (q, rf[q], r)
        assert np.allclose(sc[q], s, rtol=1e-9, atol=0)
    rf_noms, _ = device_model(g).r_factor_batch(g["N1"], g["data_c"], mask, g["idx"], X)
    assert not np.allclose(rf, rf_noms)           # the MS term is present


def test_bad_member_is_nan_and_isolated(cuda):
    g = golden("shellmodel.npz")
    sm = device_model(g)
    X = g["params"][:6].copy()
    X[2, 6] = np.nan                        # dE0 of edge 0
    X[4, 4] = np.inf                        # kmin
    rf, sc = sm.r_factor_batch(g["N1"], g["data_c"], g["mask"], g["idx"], X)
    assert np.isnan(rf[2]) and np.isnan(rf[4])
    ok = [0, 1, 3, 5]
    assert np.allclose(rf[ok], g["rf_c"][ok], rtol=1e-9, atol=0)


def test_differential_evolution_stage1(cuda):
    """The reference's global stage (per-edge dE0, sigma^2 scales, dr, C3,
    window) as differential evolution with one launch per generation: the
    result improves on the start, stays inside the bounds, and its R-factor
    equals the CPU restatement at the returned vector."""
    from chimera_b200.calibrate import Stage1, de_stage1
    g = golden("shellmodel.npz")
    sm = device_model(g)
    st = Stage1(sm, (0.5, 0.5), ms=False, free_window=True, free_dr=True, free_c3=True,
                free_shell_sigma=True, elements=("Fe", "Ni"))
    res, n = de_stage1(sm, g["N1"], g["data_c"], g["mask"], g["idx"], st, a0=3.585,
                       maxiter=15, popsize=6, seed=1, polish=False)
    start, _ = sm.r_factor_batch(g["N1"], g["data_c"], g["mask"], g["idx"],
                                 st.rows(st.x0(), a0=3.585))
    assert res.fun < start[0] and n >= 15 * 6 * len(st.names)
    lo, hi = np.array(st.bounds).T
    assert np.all(res.x >= lo) and np.all(res.x <= hi)
    row = st.rows(res.x, a0=3.585)[0]
    mask = g["mask"]
    r, _ = OS.r_factor(row, g["N1"], oracle_model(g), g["data_c"][:, mask], g["idx"][mask],
                       g["kweight"])
    assert abs(res.fun - r) <= 1e-9 * r


@pytest.mark.parametrize("tag", ["c", "m"])
def test_crlb_matches_reference(cuda, tag):
    """Cramer-Rao bounds with the default nuisances (a0, sigma^2 scale, MS
    amplitude, dE0 per edge, the free bond offsets, C3): every perturbed
    model of the finite-difference Jacobian (26 here) in one launch, then the
    FP64 Fisher matrix with the prior on the host. alpha widths, the SRO
    eigen-widths, the alpha covariance and the nuisance widths equal the
    reference's crlb to 1e-6 relative, complex and |chi(R)| data."""
    from chimera_b200.shellmodel import crlb
    g = golden("shellmodel.npz")
    sm = device_model(g)
    sm.set_flat(g["crlb_base"])
    data = g["data_c"] if tag == "c" else g["data_m"]
    r = crlb(sm, g["N1"], data, g["crlb_sigma"], g["mask"], g["idx"])
    assert r["n_models"] == 2 * (5 + 8)
    ns = r["nuisance_sd"]
    nuis = np.concatenate([np.atleast_1d(ns[k]) for k in
                           ("a0", "sigma_scale", "ms_amp", "dE0", "dr", "c3")])
    for got, key in ((r["alpha_sd"], "alpha_sd"), (r["eig_sd"], "eig_sd"),
                     (r["alpha_cov"], "alpha_cov"), (nuis, "nuis"),
                     (r["dr_entry_sd"], "dr_entry_sd")):
        ref = g[f"crlb_{tag}_{key}"]
        assert np.allclose(np.asarray(got), ref, rtol=1e-6, atol=0), (key, got, ref)
    assert np.array_equal(sm.flat(), g["crlb_base"])       # the model is left as it was
