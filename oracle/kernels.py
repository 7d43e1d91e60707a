"""ctypes bindings to oracle/chx_oracle.c (test infrastructure: the checker).

Each wrapper takes NumPy arrays in the reference kernel's argument order
(exafs_gpu/kernels.py) and writes its outputs in place, like the CuPy
RawKernel it restates. `build()` compiles the library with gcc into
oracle/_build/.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "chx_oracle.c")
_OUT = os.path.join(_HERE, "_build", "liboracle.so")
_LIB = None


def build(force=False):
    """Compile chx_oracle.c (plain C, -O2, no fast-math: FP64 is the point)."""
    if force or not os.path.exists(_OUT) or os.path.getmtime(_OUT) < os.path.getmtime(_SRC):
        os.makedirs(os.path.dirname(_OUT), exist_ok=True)
        tmp = _OUT + f".{os.getpid()}.tmp"
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
                               "-o", tmp, _SRC, "-lm"])
        os.replace(tmp, _OUT)
    return _OUT


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        _LIB.orc_splitmix64.restype = C.c_uint64
        _LIB.orc_splitmix64.argtypes = [C.c_uint64]
        _LIB.orc_u01.restype = C.c_double
        _LIB.orc_u01.argtypes = [C.c_uint64]
    return _LIB


def _p(a, dtype):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.dtype == dtype and a.flags.c_contiguous, \
        f"oracle wants a contiguous {dtype} array, got {getattr(a, 'dtype', type(a))}"
    return a.ctypes.data_as(C.c_void_p)


D, I, U8 = np.dtype(np.float64), np.dtype(np.int32), np.dtype(np.uint8)


def splitmix64(x):
    return int(lib().orc_splitmix64(C.c_uint64(int(x) & (2 ** 64 - 1))))


def u01(h):
    return float(lib().orc_u01(C.c_uint64(int(h))))


def compute_r(pos, iidx, jidx, shift, r, evec, npairs, natoms, nconf):
    lib().orc_compute_r(_p(pos, D), _p(iidx, I), _p(jidx, I), _p(shift, D), _p(r, D),
                        _p(evec, D), C.c_int(npairs), C.c_int(natoms), C.c_int(nconf))


def build_ptype(species, iidx, jidx, ptype, npairs, natoms, nconf, nsp):
    lib().orc_build_ptype(_p(species, I), _p(iidx, I), _p(jidx, I), _p(ptype, I),
                          C.c_int(npairs), C.c_int(natoms), C.c_int(nconf), C.c_int(nsp))


def chi_forward(r, ptype, shell, sig2, f, d, lam, k, dr, c3, s2, chi, npairs, nk, nconf,
                s02, nsp):
    lib().orc_chi_forward(_p(r, D), _p(ptype, I), _p(shell, I), _p(sig2, D), _p(f, D),
                          _p(d, D), _p(lam, D), _p(k, D), _p(dr, D), _p(c3, D), _p(s2, D),
                          _p(chi, D), C.c_int(npairs), C.c_int(nk), C.c_int(nconf),
                          C.c_double(s02), C.c_int(nsp))


def chi_delta(r_old, pt_old, shell, aff, r_new, pt_new, sig2, f, d, lam, k, dr, c3, s2,
              dchi, npairs, nk, nrep, maxaff, s02, nsp):
    lib().orc_chi_delta(_p(r_old, D), _p(pt_old, I), _p(shell, I), _p(aff, I),
                        _p(r_new, D), _p(pt_new, I), _p(sig2, D), _p(f, D), _p(d, D),
                        _p(lam, D), _p(k, D), _p(dr, D), _p(c3, D), _p(s2, D), _p(dchi, D),
                        C.c_int(npairs), C.c_int(nk), C.c_int(nrep), C.c_int(maxaff),
                        C.c_double(s02), C.c_int(nsp))


def commit_move(aff, r_new, pt_new, accept, r_old, pt_old, npairs, nrep, maxaff):
    lib().orc_commit_move(_p(aff, I), _p(r_new, D), _p(pt_new, I), _p(accept, U8),
                          _p(r_old, D), _p(pt_old, I), C.c_int(npairs), C.c_int(nrep),
                          C.c_int(maxaff))


def propose_select(species, pos, ideal, a, b, nsa, nsb, npa, isswap, natoms, nrep, seed,
                   stepc, swap_frac, disp_sigma, max_disp):
    lib().orc_propose_select(_p(species, I), _p(pos, D), _p(ideal, D), _p(a, I), _p(b, I),
                             _p(nsa, I), _p(nsb, I), _p(npa, D), _p(isswap, U8),
                             C.c_int(natoms), C.c_int(nrep), C.c_uint64(int(seed)),
                             C.c_uint64(int(stepc)), C.c_double(swap_frac),
                             C.c_double(disp_sigma), C.c_double(max_disp))


def propose_build(species, pos, nbr, rev, iidx, jidx, shift, a, b, nsa, nsb, npa, aff,
                  r_new, pt_new, natoms, ncoord, npairs, nrep, maxaff, nsp):
    lib().orc_propose_build(_p(species, I), _p(pos, D), _p(nbr, I), _p(rev, I), _p(iidx, I),
                            _p(jidx, I), _p(shift, D), _p(a, I), _p(b, I), _p(nsa, I),
                            _p(nsb, I), _p(npa, D), _p(aff, I), _p(r_new, D), _p(pt_new, I),
                            C.c_int(natoms), C.c_int(ncoord), C.c_int(npairs), C.c_int(nrep),
                            C.c_int(maxaff), C.c_int(nsp))


def commit_state(accept, a, b, nsa, nsb, npa, isswap, species, pos, natoms, nrep):
    lib().orc_commit_state(_p(accept, U8), _p(a, I), _p(b, I), _p(nsa, I), _p(nsb, I),
                           _p(npa, D), _p(isswap, U8), _p(species, I), _p(pos, D),
                           C.c_int(natoms), C.c_int(nrep))


def ms_counts(species, p_abs, p_cls, p_slot, cls_off, nsp, nblk):
    species = np.ascontiguousarray(species, np.int32)
    nrep, natoms = species.shape
    out = np.zeros((nrep, nsp * nblk))
    lib().orc_ms_counts(_p(species, I), C.c_int(nrep), C.c_int(natoms), _p(p_abs, I),
                        _p(p_cls, I), _p(p_slot, I), C.c_long(p_abs.size), _p(cls_off, I),
                        C.c_int(nsp), C.c_int(nblk), _p(out, D))
    return out


def ms_delta(species, inc, p_abs, p_cls, p_slot, npath, cls_off, nsp, nblk, a, b, nsa, nsb):
    species = np.ascontiguousarray(species, np.int32)
    nrep, natoms = species.shape
    out = np.zeros((nrep, nsp * nblk))
    lib().orc_ms_delta(_p(species, I), C.c_int(nrep), C.c_int(natoms), _p(inc, I),
                       C.c_int(inc.shape[1]), _p(p_abs, I), _p(p_cls, I), _p(p_slot, I),
                       C.c_long(npath), _p(cls_off, I), C.c_int(nsp), C.c_int(nblk),
                       _p(a, I), _p(b, I), _p(nsa, I), _p(nsb, I), _p(out, D))
    return out


def ft_window(chi, idx, frac, inside, w, nfft, norm, bins):
    chi = np.ascontiguousarray(chi, np.float64)
    lead = chi.shape[:-1]
    nk = chi.shape[-1]
    rows = int(np.prod(lead)) if lead else 1
    bins = np.ascontiguousarray(bins, np.int32)
    ore = np.zeros((rows, bins.size))
    oim = np.zeros((rows, bins.size))
    lib().orc_ft_window(_p(chi.reshape(rows, nk), D), C.c_int(rows), C.c_int(nk),
                        _p(np.ascontiguousarray(idx, np.int32), I),
                        _p(np.ascontiguousarray(frac, np.float64), D),
                        _p(np.ascontiguousarray(inside, np.float64), D),
                        _p(np.ascontiguousarray(w, np.float64), D), C.c_int(nfft),
                        C.c_double(norm), _p(bins, I), C.c_int(bins.size), _p(ore, D),
                        _p(oim, D))
    return (ore + 1j * oim).reshape(lead + (bins.size,))


def chi2(m, tm, sm, nsp, profile, nfit):
    """m (nrep, nchan, nwin) complex or real; tm, sm (nchan, nwin)."""
    cplx = np.iscomplexobj(tm)
    m = np.asarray(m)
    nrep, nchan, nwin = m.shape
    mr = np.ascontiguousarray(m.real, np.float64)
    mi = np.ascontiguousarray(m.imag if cplx else np.zeros_like(mr), np.float64)
    tr = np.ascontiguousarray(np.real(tm), np.float64)
    ti = np.ascontiguousarray(np.imag(tm) if cplx else np.zeros_like(tr), np.float64)
    s = np.ascontiguousarray(sm, np.float64)
    out = np.zeros(nrep)
    lib().orc_chi2(_p(mr, D), _p(mi, D), C.c_int(nrep), C.c_int(nchan), C.c_int(nwin),
                   _p(tr, D), _p(ti, D), _p(s, D), C.c_int(nsp), C.c_int(int(cplx)),
                   C.c_int(int(profile)), C.c_double(nfit), _p(out, D))
    return out
