"""The windowed FT contraction chx_ft_batch (A5) in its three precisions:
FP64 and FP32 SIMT tiles, split-BF16 on the tcgen05 tensor cores."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

# tolerance relative to the largest |chi(R)| of the case
TOL = {0: 1e-12, 1: 2e-6, 2: 1e-4, 3: 3e-3}


@pytest.mark.parametrize("precision", [0, 1, 2, 3])
@pytest.mark.parametrize("grid", ["model", "uniform", "shifted"])
def test_transform_matches_reference_goldens(cuda, grid, precision):
    """chi(R) of the reference's FourierTransform (first 256 bins) for every
    k grid and k weight of the goldens."""
    from chimera_b200.fourier import FourierTransform
    g = golden("fourier.npz")
    for kw in (1, 2, 3):
        key = f"{grid}_w{kw}"
        f = FourierTransform(g[key + "_k"], 3.0, 13.0, kw)
        z = f.to_R(g[key + "_chi"], bins=np.arange(256), precision=precision)
        want = g[key + "_R256"]
        assert np.abs(z - want).max() <= TOL[precision] * np.abs(want).max(), key


def test_split_bf16_batch_of_the_series_configuration(cuda):
    """4,096 spectra x 241 k points onto 200 R points (the series-point
    configuration's per-weight batch): the tensor-core contraction against the
    FP64 one, on rows that are not a multiple of the 128-row tile and a column
    count (400) that is not a multiple of 128."""
    import torch
    from chimera_b200.fourier import FourierTransform, apply_basis
    from chimera_b200.tables import uniform_k
    k = uniform_k()
    f = FourierTransform(k, 3.0, 13.0, 2, window="kaiser")
    B = f.basis(np.arange(46, 246))
    rng = np.random.default_rng(4)
    for rows in (4096, 1000):
        chi = rng.normal(0, 1, (rows, k.size)) * np.exp(-0.1 * k)[None]
        x = torch.from_numpy(chi).cuda()
        z0 = apply_basis(x, B, 0).cpu().numpy()
        z2 = apply_basis(x, B, 2).cpu().numpy()
        z1 = apply_basis(x, B, 1).cpu().numpy()
        z3 = apply_basis(x, B, 3).cpu().numpy()
        scale = np.abs(z0).max()
        e2 = np.abs(z2 - z0).max() / scale
        e1 = np.abs(z1 - z0).max() / scale
        e3 = np.abs(z3 - z0).max() / scale
        print(f"rows {rows}: split-BF16 max err {e2:.2e}, TF32 {e3:.2e}, FP32 {e1:.2e} "
              "(of max |chi(R)|)")
        assert e2 <= TOL[2] and e1 <= TOL[1] and e3 <= TOL[3]
        assert e2 < e3 / 10          # the split keeps about 16 bits, TF32 about 11
        # per-bin relative error stays small where chi(R) is not tiny
        big = np.abs(z0) > 0.05 * scale
        assert (np.abs(z2 - z0)[big] / np.abs(z0)[big]).max() <= 5e-3


@pytest.mark.parametrize("precision", [2, 3])
def test_tensor_core_batch_wider_than_one_wave(cuda, precision):
    """More output tiles than SMs, so that every CTA of the persistent
    contraction walks two or three tiles through both accumulators, and
    column counts (1,200 and 1,210 real columns) whose last tile has staged
    boxes wholly and partly past the end of chi(R), with the basis tile
    resident in shared memory (241 k points) and streamed beside chi (321 k
    points): each of three repeated calls into the same output equals the
    FP64 contraction within the precision's tolerance, bin by bin where
    chi(R) is not tiny."""
    import torch
    from chimera_b200.fourier import FourierTransform, apply_basis
    from chimera_b200.tables import uniform_k
    rng = np.random.default_rng(11)
    for rows, nb, kmax in ((4096, 600, 14.0), (6000, 605, 14.0), (4096, 600, 18.0)):
        k = uniform_k(2.0, kmax)
        f = FourierTransform(k, 3.0, 13.0, 2, window="kaiser")
        B = f.basis(np.arange(nb) % 250)
        chi = rng.normal(0, 1, (rows, k.size)) * np.exp(-0.1 * k)[None]
        x = torch.from_numpy(chi).cuda()
        z0 = apply_basis(x, B, 0).cpu().numpy()
        scale = np.abs(z0).max()
        big = np.abs(z0) > 0.05 * scale
        for _ in range(3):
            z = apply_basis(x, B, precision).cpu().numpy()
            assert np.abs(z - z0).max() <= TOL[precision] * scale, (rows, nb)
            assert (np.abs(z - z0)[big] / np.abs(z0)[big]).max() <= 50 * TOL[precision]


@pytest.mark.parametrize("precision", [2, 3])
def test_tensor_core_edge_shapes(cuda, precision):
    """Shapes at the edges of the tensor-core path: one spectrum, rows one past
    a 128-row tile, one and eight R points (2 and 16 real columns: a single
    chi(R) box clipped in both directions), a short k grid (one 32-wide K
    chunk) and nk = 257 (the smallest padded nk that streams the basis
    instead of keeping it resident): each equals the FP64 contraction within
    the precision's tolerance."""
    import torch
    from chimera_b200.fourier import apply_basis
    rng = np.random.default_rng(23)
    for rows, nk, nb in ((1, 241, 1), (129, 241, 8), (300, 20, 64), (257, 257, 100),
                         (128, 256, 128)):
        k = 2.0 + 0.05 * np.arange(nk)
        B = np.exp(-2j * np.outer(k, 0.1 + 0.03 * np.arange(nb))) * (k ** 2)[:, None] * 0.05
        chi = rng.normal(0, 1, (rows, nk)) * np.exp(-0.1 * k)[None]
        x = torch.from_numpy(chi).cuda()
        z0 = apply_basis(x, B, 0).cpu().numpy()
        z = apply_basis(x, B, precision).cpu().numpy()
        assert z.shape == (rows, nb)
        assert np.abs(z - z0).max() <= TOL[precision] * np.abs(z0).max(), (rows, nk, nb)


@pytest.mark.parametrize("precision,tol", [(2, 1e-4), (3, 3e-3)])
def test_fused_window_sums_match_fp64_transform(cuda, precision, tol):
    """The fused form (chx_ft_window_sums: the tensor-core contraction whose
    epilogue sums each row against the target instead of writing chi(R))
    against sums of the FP64 transform, on the series configuration's shape
    (k^2 Kaiser window, 241 k, 200 R points at 0.03 A) with a fit window
    inside the R range; rows not a multiple of the 128-row tile. The sums
    give the profiled scale and chi^2 of the reference (method_a_rmc.py:
    190-227) at any scale from the anchor s0; each sum's error is stated
    relative to its own scale, and the chi^2 relative to itself."""
    from chimera_b200.fourier import FourierTransform, WindowSums, apply_basis, window_sums
    from chimera_b200.tables import uniform_k
    k = uniform_k()
    f = FourierTransform(k, 3.0, 13.0, 2, window="kaiser")
    Rb = np.arange(46, 246)
    B = f.basis(Rb)
    rng = np.random.default_rng(7)
    rows = 1000
    chi = rng.normal(0, 0.05, (rows, k.size)) * np.exp(-0.01 * k ** 2) * np.sin(5.0 * k)
    chi[1::2] = chi[0] * (1.0 + rng.normal(0, 0.01, (rows // 2, 1)))   # near the target
    m64 = apply_basis(chi, B, 0)
    t = m64[0] * 1.1 + rng.normal(0, 1e-3, Rb.size) * (1 + 1j)
    w = np.where((f.R[Rb] >= 1.4) & (f.R[Rb] <= 5.0), 1.0 / 2e-3 ** 2, 0.0)
    inw = w != 0
    s0 = 1.1
    r0 = s0 * m64 - t
    want = np.stack([(m64 * t.conj()).real[:, inw].sum(1), (np.abs(m64) ** 2)[:, inw].sum(1),
                     (np.abs(r0) ** 2 * w).sum(1), ((m64 * r0.conj()).real * w).sum(1),
                     (np.abs(m64) ** 2 * w).sum(1), (np.abs(r0) ** 2)[:, inw].sum(1),
                     (m64 * r0.conj()).real[:, inw].sum(1)], -1)
    got = window_sums(chi, B, t, w, precision, s0=s0)
    assert got.shape == (rows, 7)
    scale = np.abs(want).max(0)
    assert (np.abs(got - want) / scale).max() <= tol
    # the profiled chi^2 from the anchored sums against FP64's own
    s64 = want[:, 0] / want[:, 1]
    c64 = (np.abs(s64[:, None] * m64 - t) ** 2 * w).sum(1)
    r64 = (np.abs(s64[:, None] * m64 - t) ** 2)[:, inw].sum(1)
    _, c, r = WindowSums.chi2(got, s0)
    near = slice(1, None, 2)                  # the rows near the target (chi^2 small)
    assert (np.abs(c - c64) / c64).max() <= 10 * tol
    assert (np.abs(c[near] - c64[near]) / c64[near]).max() <= 10 * tol
    assert (np.abs(r - r64) / r64).max() <= 10 * tol
