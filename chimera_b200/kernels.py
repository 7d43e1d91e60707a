"""The reference kernel module's interface (exafs_gpu/kernels.py:663-686).

`get(name, nsp)` returns an object called as the reference calls its CuPy
RawKernels, `k(grid, block, args, shared_mem=0)`, with the reference's
argument tuple: device arrays (anything with `data_ptr()`, e.g. torch CUDA
tensors) followed by numpy integer / float scalars. It forwards to the
matching C entry point of libchimera_b200; grid, block and shared_mem are
accepted and ignored, because the library sizes its own launches.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

# reference kernel -> (C entry, number of leading pointer arguments, scalar kinds)
_KERNELS = {
    "compute_r": ("chx_compute_r", 6, "iii"),
    "build_ptype": ("chx_build_ptype", 4, "iii"),
    "chi_forward": ("chx_chi_forward", 12, "iiid"),
    "chi_delta": ("chx_chi_delta", 15, "iiiid"),
    "commit_move": ("chx_commit_move", 6, "iii"),
    "propose_select": ("chx_propose_select", 9, "iiuuddd"),
    "propose_build": ("chx_propose_build", 15, "iiiii"),
    "commit_state": ("chx_commit_state", 9, "ii"),
}
# entries that take the species count (the reference's -DNSP) after the scalars
_TAKES_NSP = {"build_ptype", "chi_forward", "chi_delta", "propose_build"}


def _ptr(x):
    if x is None:
        return None
    return C.c_void_p(int(x.data_ptr()))


class Kernel:
    def __init__(self, name, nsp):
        if name not in _KERNELS:
            raise NotImplementedError(
                f"kernel {name!r} is not on the hot path this library implements "
                f"(available: {sorted(_KERNELS)})")
        self.name, self.nsp = name, int(nsp)
        self.entry, self.nptr, self.kinds = _KERNELS[name]

    def __call__(self, grid, block, args, shared_mem=0):
        args = list(args)
        ptrs = [_ptr(a) for a in args[:self.nptr]]
        scal = []
        for kind, v in zip(self.kinds, args[self.nptr:]):
            if kind == "i":
                scal.append(int(v))
            elif kind == "u":
                scal.append(C.c_uint64(int(np.uint64(v))))
            else:
                scal.append(float(v))
        if len(scal) != len(self.kinds):
            raise TypeError(f"{self.name}: expected {self.nptr} arrays and "
                            f"{len(self.kinds)} scalars, got {len(args)} arguments")
        extra = [self.nsp] if self.name in _TAKES_NSP else []
        N.call(self.entry, *ptrs, *scal, *extra, N.stream())


def module(nsp):
    nsp = int(nsp)
    if nsp < 2:
        raise ValueError("need at least two species")
    N.lib()
    return nsp


def get(name, nsp):
    module(nsp)
    return Kernel(name, nsp)
