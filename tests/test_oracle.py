"""The oracle is pinned to the reference's own outputs: the path sum to
ForwardModel.chi_reference, the transform to FourierTransform(xp=np), and the
product's transform set-up to the reference's arrays."""
import numpy as np
import pytest

from conftest import golden
from oracle import kernels as K
from oracle import sampler as OS


def test_splitmix_known_values():
    # the first outputs of the published splitmix64 generator seeded with 0:
    # state_i = i * golden gamma, output = mix(state_i + gamma)
    g = 0x9E3779B97F4A7C15
    out = [K.splitmix64((i * g) % 2 ** 64) for i in range(3)]
    assert out == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]
    assert K.u01(2 ** 64 - 1) < 1.0 and K.u01(2 ** 11) == 2.0 ** -53


@pytest.mark.parametrize("which", ["chi_plain", "chi_cumulant"])
def test_oracle_path_sum_matches_reference(which):
    g = golden("forward.npz")
    nsp = g["f"].shape[0]
    nconf, natoms = g["species"].shape
    npairs = g["i"].size
    nshell = int(g["shell"].max()) + 1
    cum = which == "chi_cumulant"
    dr = g["dr"].reshape(-1) if cum else np.zeros(nshell * nsp * nsp)
    c3 = g["c3"] if cum else np.zeros(nshell)
    s2 = g["s2types"].reshape(-1) if cum else np.zeros(nshell * nsp * nsp)
    r = np.zeros((nconf, npairs))
    pt = np.zeros((nconf, npairs), np.int32)
    K.compute_r(np.ascontiguousarray(g["pos"]), g["i"], g["j"], g["shift"], r, None, npairs,
                natoms, nconf)
    K.build_ptype(g["species"], g["i"], g["j"], pt, npairs, natoms, nconf, nsp)
    chi = np.zeros((nconf, nsp, g["k"].size))
    K.chi_forward(r, pt, g["shell"], g["sig2"], g["f"], np.ascontiguousarray(g["delta"].reshape(nsp * nsp, -1)),
                  g["lam"], g["k"], np.ascontiguousarray(dr), np.ascontiguousarray(c3),
                  np.ascontiguousarray(s2), chi, npairs, g["k"].size, nconf, float(g["s02"]), nsp)
    cnt = np.stack([(g["species"] == s).sum(1) for s in range(nsp)], 1)
    chi /= np.maximum(cnt, 1)[:, :, None]
    ref = g[which]
    assert np.abs(chi - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("grid", ["model", "uniform", "shifted"])
@pytest.mark.parametrize("kw", [1, 2, 3])
def test_oracle_transform_matches_reference(grid, kw):
    g = golden("fourier.npz")
    key = f"{grid}_w{kw}"
    st = OS.ft_setup(g[key + "_k"], 3.0, 13.0, kw)
    for a, b in (("idx", "_idx"), ("frac", "_frac"), ("inside", "_inside"), ("w", "_w")):
        assert np.array_equal(st[a], g[key + b]), a
    ch = OS.Channel(st["idx"], st["frac"], st["inside"], st["w"], st["nfft"], st["norm"], 0)
    z = ch.to_R(g[key + "_chi"])[:, :256]
    assert np.array_equal(z, g[key + "_R256"])
    # the direct DFT on chosen bins agrees to rounding
    bins = np.arange(0, 256, 7)
    zd = K.ft_window(g[key + "_chi"], st["idx"], st["frac"], st["inside"], st["w"], 2048,
                     st["norm"], bins)
    assert np.abs(zd - g[key + "_R256"][:, bins]).max() < 1e-12 * np.abs(g[key + "_R256"]).max()


@pytest.mark.parametrize("grid", ["model", "uniform", "shifted"])
def test_product_transform_setup_equals_reference(grid):
    from chimera_b200.fourier import FourierTransform, r_grid
    g = golden("fourier.npz")
    for kw in (1, 2, 3):
        key = f"{grid}_w{kw}"
        f = FourierTransform(g[key + "_k"], 3.0, 13.0, kw)
        assert np.array_equal(f._idx, g[key + "_idx"])
        assert np.array_equal(f._frac, g[key + "_frac"])
        assert np.array_equal(f._inside, g[key + "_inside"])
        assert np.array_equal(f._w, g[key + "_w"])
        assert f._norm == float(g[key + "_norm"])
        # the folded basis reproduces the reference transform (host check of the matrix)
        B = f.basis(np.arange(256))
        z = g[key + "_chi"] @ B
        assert np.abs(z - g[key + "_R256"]).max() < 1e-12 * np.abs(g[key + "_R256"]).max()
    assert np.array_equal(r_grid(), g["R"])


def test_oracle_chi2_profile_and_magnitude():
    rng = np.random.default_rng(0)
    m = rng.normal(size=(3, 6, 10)) + 1j * rng.normal(size=(3, 6, 10))
    t = rng.normal(size=(6, 10)) + 1j * rng.normal(size=(6, 10))
    s = np.full((6, 10), 0.5)
    c2 = K.chi2(m, t, s, 2, True, 10 * 6 * 2)
    # direct restatement of method_a_rmc.py:190-227
    num = (m.real * t.real + m.imag * t.imag).sum(-1).reshape(3, 2, 3).sum(-1)
    den = (np.abs(m) ** 2).sum(-1).reshape(3, 2, 3).sum(-1)
    sc = np.repeat(num / den, 3, axis=1)
    d = (m * sc[:, :, None] - t) / s
    assert np.allclose(c2, (np.abs(d) ** 2).sum((1, 2)) / 120, rtol=1e-14)
    c2m = K.chi2(np.abs(m), np.abs(t), s, 2, False, 60)
    d = (np.abs(m) - np.abs(t)) / s
    assert np.allclose(c2m, (d * d).sum((1, 2)) / 60, rtol=1e-14)
