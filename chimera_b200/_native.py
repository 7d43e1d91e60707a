"""ctypes binding of libchimera_b200.so (include/chimera_b200.h).

The library is the product's only compute path. Loading it fails loudly if it
is missing or cannot be built; there is no fallback. `call(name, *args)`
invokes an entry point and raises `ChxError` with the library's message on a
non-zero status. Device buffers are torch CUDA tensors passed by pointer;
`stream()` is torch's current CUDA stream, so every launch orders with torch's
own work and is captured by torch CUDA graphs.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_LIB = None


class ChxError(RuntimeError):
    pass


c_p = C.c_void_p
c_i = C.c_int
c_d = C.c_double
c_u64 = C.c_uint64
c_i64 = C.c_int64


class Pairs(C.Structure):
    """chx_pairs_t"""
    _fields_ = [("natoms", c_i), ("ncoord", c_i), ("npairs", c_i), ("nsp", c_i), ("nk", c_i),
                ("nshell", c_i),
                ("iidx", c_p), ("jidx", c_p), ("shift", c_p), ("shell", c_p), ("sig2", c_p),
                ("ftab", c_p), ("dtab", c_p), ("lamtab", c_p), ("ktab", c_p), ("drtab", c_p),
                ("c3tab", c_p), ("s2tab", c_p), ("s02", c_d)]


class Ladder(C.Structure):
    """chx_ladder_t"""
    _fields_ = [
        ("natoms", c_i), ("ncoord", c_i), ("npairs", c_i), ("nshell", c_i), ("nsp", c_i),
        ("nk", c_i),
        ("iidx", c_p), ("jidx", c_p), ("rev", c_p), ("shift", c_p), ("shell", c_p),
        ("sig2", c_p), ("pair_tab", c_p), ("ideal", c_p),
        ("ftab", c_p), ("dtab", c_p), ("lamtab", c_p), ("ktab", c_p), ("drtab", c_p),
        ("c3tab", c_p), ("s2tab", c_p), ("s02", c_d), ("sstab", c_p), ("sstab32", c_p),
        ("ms_nblk", c_i), ("ms_M", c_i), ("ms_D", c_i), ("ms_tpl", c_p), ("ms_nbr", c_p),
        ("ms_T", c_p),
        ("ms_T32", c_p),
        ("etab", c_p), ("energy_beta", c_d),
        ("nchan", c_i), ("nkw", c_i), ("nwin", c_i), ("nfft", c_i), ("ncoef", c_i),
        ("ft_n0", c_p), ("ft_idx", c_p), ("ft_frac", c_p), ("ft_w", c_p), ("win_bin", c_p),
        ("chi_extra", c_p), ("ft_norm", c_d),
        ("tm_re", c_p), ("tm_im", c_p), ("sm", c_p), ("w2", c_p), ("tnorm", c_p),
        ("cplx", c_i), ("profile", c_i),
        ("nfit", c_d),
        ("seed", c_u64), ("swap_frac", c_d), ("disp_sigma", c_d), ("max_disp", c_d),
        ("nrep", c_i), ("slot0", c_i), ("beta_rung", c_p), ("u_stream", c_p),
        ("u_steps", c_i64),
        ("species", c_p), ("pos", c_p), ("moved", c_p), ("chi", c_p), ("chi2", c_p),
        ("count", c_p), ("rung_of", c_p), ("slot_of", c_p), ("best_chi2", c_p),
        ("best_sp", c_p), ("best_pos", c_p), ("ms_C", c_p), ("acc_rung", c_p), ("acc_log", c_p), ("n_acc", c_p),
        ("exch_att", c_p), ("exch_acc", c_p),
        ("mlp", c_p), ("feat_nbr", c_p), ("feat_D", c_i), ("da_on", c_p), ("da_stat", c_p),
        ("log_codes", c_p), ("log_y", c_p), ("log_cap", c_i64), ("best_stale", c_p),
        ("xr", c_p), ("tie_eps", c_d), ("tie_stat", c_p), ("tie_gdiag", c_p), ("xs", c_p), ("ft_frag", c_p), ("ft_mt", c_i), ("ft_kt", c_i)]


class Mlp(C.Structure):
    """chx_mlp_t"""
    _fields_ = [("nsp", c_i), ("D", c_i), ("H", c_i), ("nin", c_i),
                ("W1", c_p), ("W2", c_p), ("W3", c_p), ("w4", c_p),
                ("b1", c_p), ("b2", c_p), ("b3", c_p), ("b4", c_p),
                ("out_scale", C.c_float), ("feat_shift", C.c_float), ("feat_scale", C.c_float),
                ("nchain", c_i)]


class Shell(C.Structure):
    """chx_shell_t"""
    _fields_ = [("nsp", c_i), ("nshell", c_i), ("nk", c_i), ("nkw", c_i), ("nbin", c_i),
                ("nfft", c_i), ("magnitude", c_i),
                ("a0_ref", c_d), ("s02", c_d), ("dk_win", c_d), ("dk", c_d), ("etok", c_d),
                ("k", c_p), ("f", c_p), ("delta", c_p), ("lam", c_p), ("shells_ref", c_p),
                ("sigma2_ref", c_p), ("shell_mult", c_p), ("N", c_p), ("kweight", c_p),
                ("bins", c_p), ("data", c_p),
                ("npath", c_i), ("ms_dnn", c_d), ("ms_abs", c_p), ("ms_reff", c_p),
                ("ms_deg", c_p), ("ms_F", c_p), ("ms_D", c_p), ("ms_L", c_p),
                ("N_member", c_p), ("resid", c_p), ("sigma", c_p), ("profile", c_i)]


class PathSet(C.Structure):
    """chx_path_t"""
    _fields_ = [("npath", c_i), ("maxs", c_i), ("ne", c_i), ("ntype", c_i), ("nlt", c_i),
                ("glmax", c_i), ("nsc", c_p), ("typ", c_p), ("leg", c_p), ("eul", c_p),
                ("p", c_p), ("t", c_p), ("lmax", c_p), ("goff", c_p), ("gcnt", c_p),
                ("glpp", c_p), ("gA", c_p), ("doff", c_p), ("dflat", c_p)]


# argument types of every entry point, in header order
_SIGS = {
    "chx_version": ([], c_i),
    "chx_struct_size": ([c_i], c_i64),
    "chx_last_error": ([C.c_char_p, c_i], c_i),
    "chx_compute_r": ([c_p] * 6 + [c_i] * 3 + [c_p], c_i),
    "chx_build_ptype": ([c_p] * 4 + [c_i] * 4 + [c_p], c_i),
    "chx_chi_forward": ([c_p] * 12 + [c_i] * 3 + [c_d, c_i, c_p], c_i),
    "chx_chi_delta": ([c_p] * 15 + [c_i] * 4 + [c_d, c_i, c_p], c_i),
    "chx_commit_move": ([c_p] * 6 + [c_i] * 3 + [c_p], c_i),
    "chx_propose_select": ([c_p] * 9 + [c_i, c_i, c_u64, c_u64, c_d, c_d, c_d, c_p], c_i),
    "chx_propose_build": ([c_p] * 15 + [c_i] * 6 + [c_p], c_i),
    "chx_commit_state": ([c_p] * 9 + [c_i, c_i, c_p], c_i),
    "chx_chi_full_scratch_bytes": ([c_p, c_i], c_i64),
    "chx_chi_full": ([c_p, c_p, c_p, c_i, c_i, c_p, c_p, c_i64, c_p], c_i),
    "chx_chi_full_noalloc_max_bytes": ([], c_i64),
    "chx_chi_full_noalloc": ([c_p, c_p, c_p, c_i, c_i, c_p, c_p], c_i),
    "chx_ms_counts": ([c_p, c_i, c_i, c_p, c_i64, c_i, c_i, c_p, c_p], c_i),
    "chx_ms_delta": ([c_p, c_i, c_i, c_p, c_i, c_i, c_i, c_p, c_p, c_p, c_p, c_p, c_p], c_i),
    "chx_eval_chi2": ([c_p, c_p, c_i, c_p, c_i, c_i, c_p, c_p, c_p, c_p], c_i),
    "chx_ms_chi_of": ([c_p, c_p, c_i, c_i, c_i, c_i, c_p, c_p], c_i),
    "chx_sampler_smem_bytes": ([c_p, c_i, c_i], c_i),
    "chx_shell_table": ([c_p, c_p, c_p, c_p, c_p], c_i),
    "chx_sampler_step": ([c_p, c_p, c_i, c_p, c_i, c_i, c_i, c_i, c_i, c_p, c_p, c_p, c_p], c_i),
    "chx_ft_window_sums_scratch_bytes": ([c_i, c_i, c_i, c_i], C.c_int64),
    "chx_ft_window_sums": ([c_p, c_i, c_i, c_p, c_i, c_p, c_p, c_d, c_i, c_p, c_p, C.c_int64,
                            c_p], c_i),
    "chx_pair_counts": ([c_p, c_i, c_i, c_p, c_p, c_i, c_i, c_p, c_p, c_p], c_i),
    "chx_refresh_chi2": ([c_p, c_p, c_i, c_p, c_i, c_i, c_p, c_p], c_i),
    "chx_reanchor_scratch_bytes": ([c_p, c_i, c_i], C.c_int64),
    "chx_reanchor": ([c_p, c_p, c_i, c_p, c_i, c_p, c_p, C.c_int64, c_p, c_p], c_i),
    "chx_reanchor_due": ([c_p, c_p, c_i, c_p, c_i, c_i, c_i, c_i, c_p, c_p, c_p, C.c_int64, c_p,
                          c_p], c_i),
    "chx_replica_exchange": ([c_p, c_i, c_p, c_p], c_i),
    "chx_apply_exchange": ([c_p, c_i, c_p, c_p], c_i),
    "chx_ft_batch": ([c_p, c_i, c_i, c_p, c_i, c_i, c_p, c_p, c_i64, c_p], c_i),
    "chx_ft_batch_scratch_bytes": ([c_i, c_i, c_i, c_i], c_i64),
    "chx_mlp_nparam": ([c_i, c_i, c_i, c_i], c_i64),
    "chx_mlp_bind": ([c_p, c_i, c_i, c_i, c_i, c_p, c_p], c_i),
    "chx_mlp_predict": ([c_p, c_p, c_p, c_p, c_i, c_p, c_p], c_i),
    "chx_mlp_work_bytes": ([c_i, c_i], c_i64),
    "chx_mlp_grad": ([c_p] * 5 + [c_i] + [c_p] * 5, c_i),
    "chx_mlp_adam": ([c_p] * 5 + [c_i64, C.c_float, C.c_float, C.c_float, C.c_float, c_i, c_p],
                     c_i),
    "chx_shell_nparam": ([c_i, c_i], c_i),
    "chx_shell_rfactor": ([c_p, c_p, c_i, c_p, c_p, c_p], c_i),
    "chx_path_trace": ([c_p, c_p, c_p], c_i),
}

# entry points declared in include/chimera_b200.h (checked by the tests)
EXPORTS = tuple(_SIGS)


def lib():
    """Load (building first if needed) the in-tree libchimera_b200.so."""
    global _LIB
    if _LIB is None:
        path = _build.LIB
        if _build.stale():
            try:
                path = _build.build()
            except Exception as e:          # no nvcc, or a compile error
                if not os.path.exists(path):
                    raise ChxError(f"libchimera_b200.so is missing and could not be built: {e}")
        L = C.CDLL(path)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _LIB = L
        _check_abi(L)
    return _LIB


def _check_abi(L):
    got = tuple(L.chx_struct_size(q) for q in range(8))
    want = (C.sizeof(Pairs), C.sizeof(Ladder), Ladder.exch_acc.offset, Ladder.seed.offset,
            C.sizeof(Mlp), Ladder.log_cap.offset, C.sizeof(Shell), C.sizeof(PathSet))
    if got != want:
        raise ChxError(f"ABI mismatch between chimera_b200.h and the binding: {got} != {want}")


def last_error():
    buf = C.create_string_buffer(512)
    lib().chx_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def call(name, *args):
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise ChxError(f"{name} failed ({rc}): {last_error()}")
    return rc


def stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "device buffers must be contiguous CUDA tensors"
    return C.c_void_p(t.data_ptr())


def dptr(t):
    """Integer device address (for ctypes struct fields)."""
    return 0 if t is None else int(t.data_ptr())


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise ChxError("chimera_b200 needs a CUDA device (sm_100a); none is visible")
    lib()


def to_dev(a, dtype=None):
    """numpy -> contiguous CUDA tensor (dtype kept unless given)."""
    import torch
    a = np.ascontiguousarray(a if dtype is None else np.asarray(a, dtype=dtype))
    return torch.from_numpy(a).to("cuda")
