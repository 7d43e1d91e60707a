"""NumPy-backed stand-in for `cupy`, used only by tests/golden/make_golden.py.

It lets the reference's own Python modules (which `import cupy`) run in this
container with no GPU, so that golden vectors come from the reference code
itself. Array calls go to NumPy; `RawModule` returns the C oracle's
restatements of the reference's NVRTC kernels (oracle/kernels.py), called
with the reference's own argument tuples. Test infrastructure only.
"""
import re as _re
import sys as _sys
import types as _types

import numpy as _np

ndarray = _np.ndarray


def __getattr__(name):
    return getattr(_np, name)


def asnumpy(x, *a, **k):
    return _np.asarray(x)


def asarray(x, dtype=None, order=None):
    return _np.asarray(x, dtype=dtype, order=order)


def ascontiguousarray(x, dtype=None):
    return _np.ascontiguousarray(x, dtype=dtype)


class _Null:
    @staticmethod
    def synchronize():
        return None


class _Stream:
    null = _Null()


cuda = _types.SimpleNamespace(Stream=_Stream)
random = _types.SimpleNamespace(default_rng=_np.random.default_rng)
fft = _np.fft
linalg = _np.linalg


def _scalar(x):
    if isinstance(x, (_np.integer, int)):
        return int(x)
    if isinstance(x, (_np.floating, float)):
        return float(x)
    return x


class _Kernel:
    def __init__(self, name, nsp):
        self.name, self.nsp = name, nsp

    def __call__(self, grid, block, args, shared_mem=0):
        from oracle import kernels as K
        a = [_scalar(x) for x in args]
        n = self.name
        if n == "compute_r":
            K.compute_r(*a)
        elif n == "build_ptype":
            K.build_ptype(*a, self.nsp)
        elif n == "chi_forward":
            K.chi_forward(*a, self.nsp)
        elif n == "chi_delta":
            K.chi_delta(*a, self.nsp)
        elif n == "commit_move":
            K.commit_move(*a)
        elif n == "propose_select":
            K.propose_select(*a)
        elif n == "propose_build":
            K.propose_build(*a, self.nsp)
        elif n == "commit_state":
            K.commit_state(*a)
        else:
            raise NotImplementedError(f"oracle has no restatement of kernel {n!r}")


class RawModule:
    def __init__(self, code=None, options=(), backend=None, **kw):
        m = [_re.match(r"-DNSP=(\d+)", o) for o in options]
        m = [x for x in m if x]
        self.nsp = int(m[0].group(1)) if m else None

    def get_function(self, name):
        return _Kernel(name, self.nsp)
