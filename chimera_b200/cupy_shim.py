"""A `cupy` importable by the reference's unchanged callers, backed by torch.

The reference's model wiring and multi-edge transform (`chimera/model.py:81`,
`chimera/multift.py:20`) and its supercell MS (`chimera/mslibrary.py`)
`import cupy` and use a small part of its array API on the arrays this
package returns. `install()` registers this module as `cupy` (and
`cupy.cuda`) so those files import and run unchanged next to chimera_b200:
device arrays are torch CUDA tensors, the same objects the package's classes
take and return. It is an import adapter for exactly that surface:

  asarray, asnumpy, abs, maximum, stack, zeros, arange, bincount,
  broadcast_to, concatenate, where, float64, int32, ndarray,
  cuda.Stream.null.synchronize

and nothing else. There is no CPU path: creating a device array without a
CUDA device raises.
"""
from __future__ import annotations

import sys
import types

import numpy as np

_TORCH = None


def _torch():
    global _TORCH
    if _TORCH is None:
        import torch
        _TORCH = torch
    return _TORCH


def _dtype(dt):
    """numpy / Python / torch dtype -> torch dtype (None stays None)."""
    torch = _torch()
    if dt is None or isinstance(dt, torch.dtype):
        return dt
    return {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
            np.dtype(np.int64): torch.int64, np.dtype(np.int32): torch.int32,
            np.dtype(np.uint8): torch.uint8, np.dtype(np.bool_): torch.bool,
            np.dtype(np.complex128): torch.complex128,
            np.dtype(np.complex64): torch.complex64}[np.dtype(dt)]


def _device():
    torch = _torch()
    if not torch.cuda.is_available():
        raise RuntimeError("the cupy adapter of chimera_b200 needs a CUDA device")
    return "cuda"


def _t(x):
    torch = _torch()
    return x if isinstance(x, torch.Tensor) else asarray(x)


# ------------------------------------------------------------------ the surface
def asarray(a, dtype=None):
    torch = _torch()
    if isinstance(a, torch.Tensor):
        t = a.to(_device())
        return t if dtype is None else t.to(_dtype(dtype))
    arr = np.asarray(a)
    t = torch.from_numpy(np.ascontiguousarray(arr)).to(_device())
    return t if dtype is None else t.to(_dtype(dtype))


def asnumpy(a):
    torch = _torch()
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def abs(a):   # noqa: A001 - the cupy name
    return _torch().abs(_t(a))


def maximum(a, b):
    torch = _torch()
    a_t = isinstance(a, torch.Tensor)
    b_t = isinstance(b, torch.Tensor)
    if a_t and not b_t:
        b = torch.as_tensor(b, dtype=a.dtype, device=a.device)
    elif b_t and not a_t:
        a = torch.as_tensor(a, dtype=b.dtype, device=b.device)
    elif not a_t and not b_t:
        a, b = asarray(a), asarray(b)
    return torch.maximum(a, b)


def stack(arrays, axis=0):
    return _torch().stack([_t(a) for a in arrays], dim=axis)


def concatenate(arrays, axis=0):
    return _torch().cat([_t(a) for a in arrays], dim=axis)


def zeros(shape, dtype=float):
    return _torch().zeros(shape, dtype=_dtype(dtype), device=_device())


def arange(*args, dtype=None):
    torch = _torch()
    return torch.arange(*args, device=_device(),
                        dtype=_dtype(dtype) if dtype is not None else None)


def bincount(x, weights=None, minlength=0):
    torch = _torch()
    return torch.bincount(_t(x).long(), weights=None if weights is None else _t(weights),
                          minlength=int(minlength))


def broadcast_to(a, shape):
    return _t(a).expand(*shape) if isinstance(shape, (tuple, list)) else _t(a).expand(shape)


def where(cond, a, b):
    torch = _torch()
    cond = _t(cond)
    if not isinstance(a, torch.Tensor):
        a = torch.as_tensor(a, device=cond.device)
    if not isinstance(b, torch.Tensor):
        b = torch.as_tensor(b, device=cond.device)
    return torch.where(cond, a, b)


float64 = np.float64
int32 = np.int32


class _NdarrayMeta(type):
    def __instancecheck__(cls, obj):
        return isinstance(obj, _torch().Tensor)


class ndarray(metaclass=_NdarrayMeta):
    """isinstance(x, cupy.ndarray) is true for torch tensors."""


class _NullStream:
    @staticmethod
    def synchronize():
        _torch().cuda.synchronize()


class _Stream:
    null = _NullStream()


cuda = types.ModuleType("cupy.cuda")
cuda.Stream = _Stream


def install():
    """Register this adapter as `cupy` (and `cupy.cuda`) in sys.modules,
    replacing any module of that name, and return it."""
    mod = sys.modules[__name__]
    sys.modules["cupy"] = mod
    sys.modules["cupy.cuda"] = cuda
    return mod


SURFACE = ("asarray", "asnumpy", "abs", "maximum", "stack", "zeros", "arange", "bincount",
           "broadcast_to", "concatenate", "where", "float64", "int32", "ndarray", "cuda")
