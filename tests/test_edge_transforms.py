"""The package's multi-edge channel set (fourier.EdgeTransforms) against the
reference's own adapter, chimera/multift.py:34-63, run by the golden script
over the reference's FourierTransform(xp=np): two edges on different k axes
(the model grid and an E0-shifted one), k^1/k^2/k^3, with a fixed chi_extra."""
import numpy as np
import pytest

from conftest import golden


def _channels(g):
    from chimera_b200.fourier import EdgeTransforms
    return EdgeTransforms.build([g["model_w1_k"], g["shifted_w1_k"]], 3.0, 13.0, (1, 2, 3),
                                chi_extra=g["multi_extra"])


def test_channel_layout_matches_reference_adapter():
    g = golden("fourier.npz")
    ft = _channels(g)
    assert ft.nchan == 6 and ft.nsp == 2
    assert np.array_equal(ft.chan_edge, np.repeat(np.arange(2), 3))
    assert np.array_equal(ft.R, g["R"])
    assert np.array_equal(ft.window_mask(1.4, 5.0), g["mask_14_50"])


def test_edge_bases_reproduce_reference_transform():
    """The per-edge bases applied on the host (the same linear map the device
    contraction applies) give the reference adapter's chi(R)."""
    g = golden("fourier.npz")
    ft = _channels(g)
    chi = g["multi_chi"] + g["multi_extra"]
    bins = np.arange(256)
    got = np.concatenate([(chi[:, e, :] @ ft.edge_basis(e, bins)).reshape(chi.shape[0], 3, 256)
                          for e in range(2)], axis=1)
    want = g["multi_R256"]
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.gpu
def test_edge_transforms_on_device_match_reference_adapter(cuda):
    g = golden("fourier.npz")
    ft = _channels(g)
    z = ft.to_R(g["multi_chi"], bins=np.arange(256))
    want = g["multi_R256"]
    assert isinstance(z, np.ndarray) and z.shape == want.shape
    assert np.abs(z - want).max() <= 1e-12 * np.abs(want).max()
