"""The C-ABI library loads without a GPU and exports every declared entry."""
import ctypes
import os
import re

from conftest import ROOT


def header_names():
    src = open(os.path.join(ROOT, "include", "chimera_b200.h")).read()
    return set(re.findall(r"^CHX_API\s+\w+\s+(chx_\w+)\s*\(", src, flags=re.M))


def test_library_exports_every_declared_symbol():
    from chimera_b200 import _native as N
    lib = N.lib()
    names = header_names()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the binding's signature table covers the header exactly
    assert names == set(N.EXPORTS)


def test_struct_layout_matches_binding():
    from chimera_b200 import _native as N
    lib = N.lib()
    assert lib.chx_struct_size(0) == ctypes.sizeof(N.Pairs)
    assert lib.chx_struct_size(1) == ctypes.sizeof(N.Ladder)
    assert lib.chx_struct_size(2) == N.Ladder.exch_acc.offset
    assert lib.chx_struct_size(3) == N.Ladder.seed.offset
    assert lib.chx_struct_size(4) == ctypes.sizeof(N.Mlp)
    assert lib.chx_struct_size(5) == N.Ladder.log_cap.offset
    assert lib.chx_version() >= 1000


def test_errors_are_reported_not_raised_in_c():
    from chimera_b200 import _native as N
    lib = N.lib()
    rc = lib.chx_compute_r(None, None, None, None, None, None, 0, 0, 0, None)
    assert rc == -1
    assert "compute_r" in N.last_error()
    rc = lib.chx_chi_full_scratch_bytes(None, 1)
    assert rc == -1


def test_surrogate_entries_check_their_arguments():
    """Shapes and alignment are checked before anything reaches the device."""
    from chimera_b200 import _native as N
    from oracle import mlp as OM
    lib = N.lib()
    for nsp, D, nchain, H in ((2, 42, 512, 256), (3, 12, 0, 64), (4, 8, 7, 8)):
        nin = OM.nin_of(nsp, D, nchain)
        assert lib.chx_mlp_nparam(nsp, D, nchain, H) == (nin + 1) * H + 3 * H + 2 * H * H + H + 1
    for bad in ((1, 42, 0, 256), (2, 0, 0, 256), (2, 42, 0, 260), (2, 42, 0, 264), (2, 128, 0, 64)):
        assert lib.chx_mlp_nparam(*bad) == -1
    P = N.Mlp()
    rc = lib.chx_mlp_bind(ctypes.byref(P), 2, 42, 0, 256, ctypes.c_void_p(4096),
                          ctypes.c_void_p(4096 + 8))
    assert rc == -1 and "16-byte" in N.last_error()
    rc = lib.chx_mlp_bind(ctypes.byref(P), 2, 42, 0, 256, ctypes.c_void_p(4096),
                          ctypes.c_void_p(8192))
    assert rc == 0 and P.nin == OM.nin_of(2, 42) and P.H == 256 and P.nchain == 0
    assert lib.chx_mlp_predict(None, None, None, None, 1, None, None) == -1
    assert lib.chx_mlp_adam(None, None, None, None, None, 1, 1e-3, .9, .999, 1e-8, 0, None) == -1


def test_tensor_core_transform_sizes_its_scratch():
    """Precisions 2 (split-BF16) and 3 (TF32) need a scratch of the basis
    and chi operand parts plus an error word, and a 16-byte aligned output;
    a smaller scratch or a misaligned output is refused with a message."""
    from chimera_b200 import _native as N
    lib = N.lib()
    rows, nk, nR = 4096, 241, 200
    Mp, Np, Kp = -(-rows // 128) * 128, -(-2 * nR // 128) * 128, -(-nk // 32) * 32
    assert lib.chx_ft_batch_scratch_bytes(rows, nk, nR, 2) == 256 + 2 * (Mp + Np) * Kp * 2
    assert lib.chx_ft_batch_scratch_bytes(rows, nk, nR, 3) == 256 + (Mp + Np) * Kp * 4
    assert lib.chx_ft_batch_scratch_bytes(rows, nk, nR, 0) == 0
    fake = ctypes.c_void_p(1 << 20)
    for prec in (2, 3):
        need = lib.chx_ft_batch_scratch_bytes(rows, nk, nR, prec)
        rc = lib.chx_ft_batch(fake, rows, nk, fake, nR, prec, fake, fake, need - 1, None)
        assert rc == -1 and "scratch" in N.last_error()
        # chi(R) is written by TMA tensor stores: out must be 16-byte aligned
        odd = ctypes.c_void_p((1 << 20) + 8)
        rc = lib.chx_ft_batch(fake, rows, nk, fake, nR, prec, odd, fake, need, None)
        assert rc == -1 and "16-byte" in N.last_error()
    assert lib.chx_ft_batch(fake, rows, nk, fake, nR, 7, fake, fake, 0, None) == -1


def test_calibration_and_path_trace_entries_check_their_arguments():
    """chx_shell_rfactor and chx_path_trace reject bad descriptors with a
    message before touching the device (no GPU needed); their structs match
    the binding."""
    import ctypes as C
    from chimera_b200 import _native as N
    lib = N.lib()
    assert lib.chx_struct_size(6) == C.sizeof(N.Shell)
    assert lib.chx_struct_size(7) == C.sizeof(N.PathSet)
    assert lib.chx_shell_nparam(2, 5) == 33 and lib.chx_shell_nparam(3, 3) == 39
    assert lib.chx_shell_nparam(0, 5) == -1
    S = N.Shell()
    S.nsp, S.nshell, S.nk, S.nkw, S.nbin, S.nfft, S.dk, S.dk_win = 2, 5, 241, 3, 100, 2048, 0.05, 1.0
    dummy = C.c_void_p(16)
    rc = lib.chx_shell_rfactor(C.byref(S), dummy, 4, dummy, dummy, None)
    assert rc == -1 and "NULL" in N.last_error()
    S.nfft = 1000                                    # not a power of two
    rc = lib.chx_shell_rfactor(C.byref(S), dummy, 4, dummy, dummy, None)
    assert rc == -1 and "limits" in N.last_error()
    P = N.PathSet()
    P.npath, P.maxs, P.ne, P.ntype, P.nlt, P.glmax = 3, 2, 10, 2, 60, 48   # lmax cap is 40
    rc = lib.chx_path_trace(C.byref(P), dummy, None)
    assert rc == -1 and "bad sizes" in N.last_error()
    P.glmax = 20
    rc = lib.chx_path_trace(C.byref(P), dummy, None)
    assert rc == -1 and "NULL" in N.last_error()
