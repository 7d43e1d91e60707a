"""The allocation-free path sum, chx_chi_full_noalloc, against chx_chi_full.

Callers that cannot allocate device memory (a host embedding the library
through a foreign-function interface with no device allocator, or code
running where allocation is not allowed) call chx_chi_full_noalloc, whose
scratch is a fixed device array inside the library. This test calls it
through the C ABI twice in a row, so the second call reuses the array the
first one left behind, and compares both results with the caller-scratch
entry point at the FP64 tolerance of the other path-sum tests. It also checks
that a request larger than the fixed array is refused.

The file sorts last so that a run stopping at the first failure has already
run every other test; it passes alone in a fresh process too.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem():
    from chimera_b200 import lattice as L
    from chimera_b200.forward import ForwardModel
    from chimera_b200.tables import smooth_tables, uniform_k
    cell = L.CrystalSupercell("fcc", (5, 5, 5), 3.59)
    top = L.Topology(cell, 5.0, sigma2=0.006)
    fm = ForwardModel(cell, smooth_tables(uniform_k(), ("Fe", "Ni")), top.i, top.j, top.shift,
                      sigma2=top.sigma2, shell=top.shell)
    rng = np.random.default_rng(11)
    nconf = 3
    sp = np.stack([L.random_config(cell.natoms, (0.5, 0.5), s) for s in range(nconf)])
    pos = np.repeat(cell.ideal[None], nconf, 0) + rng.normal(0, 0.01, (nconf, cell.natoms, 3))
    return fm, pos, sp


def test_noalloc_matches_caller_scratch_twice(cuda):
    torch = cuda
    from chimera_b200 import _native as N
    fm, pos, sp = _problem()
    P = fm.pairs_desc()
    gpos = torch.from_numpy(pos).to("cuda")
    gsp = torch.from_numpy(sp.astype(np.int32)).to("cuda")
    nconf = pos.shape[0]
    for precision, rtol in ((0, 1e-12), (1, 1e-12)):
        need = int(N.lib().chx_chi_full_scratch_bytes(ctypes.byref(P), nconf))
        assert 0 < need <= int(N.lib().chx_chi_full_noalloc_max_bytes())
        scr = torch.empty(need, dtype=torch.uint8, device="cuda")
        ref = torch.empty((nconf, fm.nsp, fm.nk), dtype=torch.float64, device="cuda")
        N.call("chx_chi_full", ctypes.byref(P), N.ptr(gpos), N.ptr(gsp), nconf, precision,
               N.ptr(ref), N.ptr(scr), need, N.stream())
        ref = ref.cpu().numpy()
        for _ in range(2):
            out = torch.full((nconf, fm.nsp, fm.nk), np.nan, dtype=torch.float64, device="cuda")
            N.call("chx_chi_full_noalloc", ctypes.byref(P), N.ptr(gpos), N.ptr(gsp), nconf,
                   precision, N.ptr(out), N.stream())
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.abs(got - ref).max() <= rtol * np.abs(ref).max()


def test_noalloc_refuses_requests_beyond_its_array(cuda):
    torch = cuda
    from chimera_b200 import _native as N
    fm, pos, sp = _problem()
    P = fm.pairs_desc()
    cap = int(N.lib().chx_chi_full_noalloc_max_bytes())
    nconf = 1        # the smallest power of two of configurations that no longer fits
    while int(N.lib().chx_chi_full_scratch_bytes(ctypes.byref(P), nconf)) <= cap:
        nconf *= 2
    gpos = torch.zeros((nconf, fm.natoms, 3), dtype=torch.float64, device="cuda")
    gsp = torch.zeros((nconf, fm.natoms), dtype=torch.int32, device="cuda")
    out = torch.zeros((nconf, fm.nsp, fm.nk), dtype=torch.float64, device="cuda")
    rc = N.lib().chx_chi_full_noalloc(ctypes.byref(P), N.ptr(gpos), N.ptr(gsp), nconf, 0,
                                      N.ptr(out), N.stream())
    assert rc == -4
    assert "fixed array" in N.last_error()


def test_noalloc_reports_device_errors_as_nan(cuda):
    """A species value outside the tables and a pair index beyond the cell are
    caught on the device (no fault): the error word lives in the library's
    array, so the call reports it as NaN in every chi value; the next good
    call on the same array is clean again (each call clears the word)."""
    torch = cuda
    from chimera_b200 import _native as N
    fm, pos, sp = _problem()
    gpos = torch.from_numpy(pos).to("cuda")
    nconf = pos.shape[0]
    good = torch.from_numpy(sp.astype(np.int32)).to("cuda")
    bad_sp = good.clone()
    bad_sp[1, 7] = fm.nsp                     # one species beyond the tables
    bad_i = fm.d_i.clone()
    bad_i[5] = fm.natoms                      # one pair index beyond the cell
    for gsp, iidx in ((bad_sp, None), (good, bad_i)):
        Pb = fm.pairs_desc()
        if iidx is not None:
            Pb.iidx = N.dptr(iidx)
        out = torch.zeros((nconf, fm.nsp, fm.nk), dtype=torch.float64, device="cuda")
        N.call("chx_chi_full_noalloc", ctypes.byref(Pb), N.ptr(gpos), N.ptr(gsp), nconf, 0,
               N.ptr(out), N.stream())
        assert torch.isnan(out).all()
        P = fm.pairs_desc()
        N.call("chx_chi_full_noalloc", ctypes.byref(P), N.ptr(gpos), N.ptr(good), nconf, 0,
               N.ptr(out), N.stream())
        assert torch.isfinite(out).all()
