"""The `cupy` import adapter for the reference's unchanged callers."""
import sys

import numpy as np
import pytest


@pytest.fixture
def cp():
    saved = {k: sys.modules.get(k) for k in ("cupy", "cupy.cuda")}
    from chimera_b200 import cupy_shim
    mod = cupy_shim.install()
    yield mod
    for k, v in saved.items():
        if v is None:
            sys.modules.pop(k, None)
        else:
            sys.modules[k] = v


def test_install_registers_the_surface(cp):
    import importlib
    import torch
    assert importlib.import_module("cupy") is cp
    assert importlib.import_module("cupy.cuda").Stream.null.synchronize
    for name in cp.SURFACE:
        assert hasattr(cp, name), name
    assert cp._dtype(np.float64) is torch.float64 and cp._dtype(cp.int32) is torch.int32
    assert cp._dtype(float) is torch.float64 and cp._dtype(np.complex128) is torch.complex128
    assert isinstance(torch.zeros(1), cp.ndarray) and not isinstance(np.zeros(1), cp.ndarray)
    if not torch.cuda.is_available():
        with pytest.raises(RuntimeError, match="CUDA"):
            cp.asarray(np.zeros(3))


@pytest.mark.gpu
def test_the_callers_expressions_on_device_arrays(cp, cuda):
    """The expressions of model.py / multift.py / SupercellMS on device
    arrays, against NumPy."""
    rng = np.random.default_rng(0)
    a, b = rng.normal(size=(3, 5)), rng.normal(size=(3, 5))
    A, B = cp.asarray(a), cp.asarray(b)
    assert isinstance(A, cp.ndarray) and A.is_cuda
    assert np.array_equal(cp.asnumpy(cp.abs(A)), np.abs(a))
    assert np.array_equal(cp.asnumpy(cp.maximum(A, 0.1)), np.maximum(a, 0.1))
    assert np.array_equal(cp.asnumpy(cp.maximum(A, B)), np.maximum(a, b))
    assert np.array_equal(cp.asnumpy(cp.stack([A, B], axis=1)), np.stack([a, b], axis=1))
    assert np.array_equal(cp.asnumpy(cp.concatenate([A, B])), np.concatenate([a, b]))
    z = cp.zeros((2, 4), dtype=cp.float64)
    assert z.dtype == cuda.float64 and z.shape == (2, 4) and z.is_cuda
    r = cp.arange(6, dtype=cp.int32)
    assert r.dtype == cuda.int32 and np.array_equal(cp.asnumpy(r), np.arange(6))
    idx = np.array([0, 3, 3, 1, 7])
    w = rng.normal(size=5)
    assert np.array_equal(cp.asnumpy(cp.bincount(cp.asarray(idx), minlength=9)),
                          np.bincount(idx, minlength=9))
    assert np.allclose(cp.asnumpy(cp.bincount(cp.asarray(idx), weights=cp.asarray(w),
                                              minlength=9)),
                       np.bincount(idx, weights=w, minlength=9), rtol=0, atol=1e-15)
    assert np.array_equal(cp.asnumpy(cp.broadcast_to(cp.asarray(a[0]), (4, 5))),
                          np.broadcast_to(a[0], (4, 5)))
    assert np.array_equal(cp.asnumpy(cp.where(A > 0, A, 0.0)), np.where(a > 0, a, 0.0))
    cp.cuda.Stream.null.synchronize()
    # the package's transform takes and returns the adapter's arrays
    from chimera_b200.fourier import FourierTransform
    from chimera_b200.tables import uniform_k
    k = uniform_k()
    f = FourierTransform(k, 3.0, 13.0, 2)
    chi = cp.asarray(rng.normal(size=(2, k.size)))
    zr = f.to_R(chi)
    assert isinstance(zr, cp.ndarray)
    assert np.allclose(cp.asnumpy(zr), f.to_R(cp.asnumpy(chi)), rtol=0, atol=1e-12)
