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
    assert lib.chx_version() >= 1000


def test_errors_are_reported_not_raised_in_c():
    from chimera_b200 import _native as N
    lib = N.lib()
    rc = lib.chx_compute_r(None, None, None, None, None, None, 0, 0, 0, None)
    assert rc == -1
    assert "compute_r" in N.last_error()
    rc = lib.chx_chi_full_scratch_bytes(None, 1)
    assert rc == -1
